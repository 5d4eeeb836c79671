// Commit kernels: weight packing + Mobius, the systematic index-two QA
// encoding by unnormalised WHTs, row-leaf BLAKE2s, and Merkle levels.
//
// Layout of one committed block (C = 32 columns, R message rows per column):
// codeword entry (c, r) at cw[c * 2R + r], message half r < R, parity half
// r >= R (qafold_short_pc.rs:461-550, `encoded_entries[col * n_ext_rows + row]`).
// A logical witness index i = c * R + r therefore lives at
//   addr(i) = (i >> logR) * 2R + (i & (R - 1))          (message half)
// and the parity of the same (c, r) at addr(i) + R.
//
// Reference algorithms: pack (packed.rs:226-243), mobius_in_place
// (packed.rs:708-752: high -= low at every level), encode index-two
// (qafold_short.rs:975-1002: parity = WHT(alpha1 * WHT(message))), leaf and
// inner hashing (qafold_short_pc.rs:2372-2517).
#pragma once
#include <cstdint>

#include "../device/blake2s_dev.cuh"
#include "../device/field_dev.cuh"
#include "../device/hash_prefix.h"

namespace QFD_NS {

__device__ __forceinline__ size_t msg_addr(size_t i, int logR) {
  return ((i >> logR) << (logR + 1)) | (i & ((size_t(1) << logR) - 1));
}
// The same in 32 bits, for the transform passes: a block's codeword holds at
// most 2^31 elements (the launchers check logm <= 30), so every index fits
// and the per-element address arithmetic takes single-word instructions.
__device__ __forceinline__ uint32_t msg_addr32(uint32_t i, int logR) {
  return ((i >> logR) << (logR + 1)) | (i & ((1u << logR) - 1u));
}

enum ButterflyOp { kMobius = 0, kWht = 1 };

// ---------------------------------------------------------------- planar tiles
// A shared-memory tile holds each of the 8 coefficients of its elements in a
// separate 32-bit plane.  Entry e of a plane sits at e ^ swz(e >> 5), an XOR
// of its bank bits with a GF(2)-linear image of bits 5..7 (columns 4, 9, 18):
// every warp access of the load/store loops and of the butterfly stages the
// passes run (radix 8 at bit offsets 0, 2 and 3, radix 2 at bit 5, and radix
// 4 at bit 4 with its groups' bits 4 and 5 swapped, see tile_loop) then hits
// 32 distinct banks.  Butterflies run in radix-8 register stages on lazily reduced
// values: a value entering level l of a pass is < 2^l * p, a difference is
// formed as a + 2^l p - b, so twelve levels stay below 2^28 and one
// reduction per pass suffices.  Both transforms act coefficient-wise over F_p.
constexpr int kTileThreads = 512;       // CTA size of the tile kernels
constexpr int kAlphaTileThreads = 512;  // the WHT tile that multiplies by alpha
constexpr int kMaxTileLog = 12;                 // 4096 elements per tile
constexpr int kPlane = 1 << kMaxTileLog;        // plane stride (words)
constexpr size_t kTileSmem = size_t(kC) * kPlane * 4;  // kC planes: 128 KiB (F65521), 64 KiB (KoalaBear)
constexpr int kCLog = kC == 8 ? 3 : 2;
__device__ __forceinline__ int pidx(int e) {
  // byte z of kSwz is swz(z); swz is linear over GF(2), so for index parts
  // with disjoint bits pidx(x | y) = pidx(x) ^ pidx(y).
  constexpr uint64_t kSwz = 0x1f1b16120d090400ull;
  return e ^ int(__byte_perm(uint32_t(kSwz), uint32_t(kSwz >> 32), (e >> 5) & 7) & 31);
}

// 16 bytes global -> shared memory, asynchronously (cp.async, L2 only).
__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src) {
  const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(src) : "memory");
}

__device__ __forceinline__ void planar_put(uint32_t* planes, int e, const Fr& v) {
  const int q = pidx(e);
#pragma unroll
  for (int c = 0; c < kC; ++c) planes[c * kPlane + q] = v.c[c];
}
// The element at plane position e, reduced to canonical form and packed.
__device__ __forceinline__ uint4 planar_get_packed(const uint32_t* planes, int e) {
  const int q = pidx(e);
  Fr v;
#pragma unroll
  for (int c = 0; c < kC; ++c) v.c[c] = tile_final(planes[c * kPlane + q]);
  return pack_fe(v);
}

// One radix-2^R register stage: levels [lvl, lvl + R) of the pass, acting on
// tile bits [b, b + R).  A work item is a group of 2^R elements and a run of
// coefficient planes (all 8, or fewer when the CTA has more threads than
// groups); its plane offsets are computed once (pidx is XOR-linear over the
// disjoint base and level bits).  Consecutive threads take consecutive groups
// of the same planes.
template <int OP, int R, bool SWAP45 = false>
__device__ __forceinline__ void planar_stage(uint32_t* planes, int log_n, int b, int lvl) {
  const int lg = log_n - R;
  int split = 0;
  while (split < kCLog && (1 << (lg + split)) < int(blockDim.x)) ++split;
  const int ppi = kC >> split;  // planes per item
  const int bmask = (1 << b) - 1;
  int off[1 << R];
#pragma unroll
  for (int j = 0; j < (1 << R); ++j) off[j] = pidx(j << b);
  for (int item = threadIdx.x; item < (1 << (lg + split)); item += blockDim.x) {
    int g = item & ((1 << lg) - 1);
    const int c0 = (item >> lg) * ppi;
    // SWAP45 (a radix-4 stage on bits 4..5 of a full tile, lg = 10): swap
    // group bits 4 and 5, a bijection of [0, 2^lg), so that a warp's groups
    // cover tile bits 0..3 and 7 (see tile_loop).
    if (SWAP45) g = (g & ~0x30) | ((g >> 1) & 0x10) | ((g << 1) & 0x20);
    const int pb = pidx((g & bmask) | ((g & ~bmask) << R));
    int q[1 << R];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) q[j] = pb ^ off[j];
#pragma unroll
    for (int cc = 0; cc < kC; ++cc) {
      if (cc >= ppi) break;
      uint32_t* pl = planes + (c0 + cc) * kPlane;
      uint32_t v[1 << R];
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) v[j] = pl[q[j]];
#pragma unroll
      for (int sft = 0; sft < R; ++sft) {
        const uint32_t B = tile_bound(lvl + sft);  // bound entering this level
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
          if (j & (1 << sft)) continue;
          if (OP == kWht) bfly_wht(v[j], v[j | (1 << sft)], B);
          else bfly_mobius(v[j], v[j | (1 << sft)], B);
        }
      }
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) pl[q[j]] = v[j];
    }
  }
  __syncthreads();
}

// Levels act on tile bits [bit0, bit0 + levels) of the 2^log_n elements; the
// first of them is level lvl0 of the pass (for the lazy bounds).
template <int OP>
__device__ __forceinline__ void planar_levels(uint32_t* planes, int log_n, int bit0, int levels, int lvl0 = 0) {
  int l = 0;
  for (; l + 3 <= levels; l += 3) planar_stage<OP, 3>(planes, log_n, bit0 + l, lvl0 + l);
  if (levels - l == 2) planar_stage<OP, 2>(planes, log_n, bit0 + l, lvl0 + l);
  if (levels - l == 1) planar_stage<OP, 1>(planes, log_n, bit0 + l, lvl0 + l);
}

// ---------------------------------------------------------------- tile passes
// A pass applies the levels on tile bits [b0, log_n) of a 2^log_n-element
// tile.  ld(t) returns the canonical value of tile element t (from HBM) and
// st(t, u) stores element t packed.  For a full 4096-element tile with at
// least three levels, the levels on tile bits 9..11 run in registers right
// after the loads (head_levels) and the last one to three levels right before
// the stores (pass_tail): a thread owns 8 (or 4, 2) elements with all 8
// coefficients, and consecutive threads take consecutive elements, so every
// load and store instruction of a warp stays coalesced.  The levels between
// run as planar shared-memory stages.  Smaller tiles run every level in
// shared memory.

// R levels across the elements held in registers, starting at level lvl.
template <int OP, int R>
__device__ __forceinline__ void reg_levels(uint32_t (&v)[1 << R][kC], int lvl) {
#pragma unroll
  for (int sft = 0; sft < R; ++sft) {
    const uint32_t B = tile_bound(lvl + sft);
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      if (j & (1 << sft)) continue;
#pragma unroll
      for (int c = 0; c < kC; ++c) {
        if (OP == kWht) bfly_wht(v[j][c], v[j | (1 << sft)][c], B);
        else bfly_mobius(v[j][c], v[j | (1 << sft)][c], B);
      }
    }
  }
}

// Levels 0..2 on tile bits 9..11 from values already loaded, into the
// planes.  Thread g (512 per CTA) owns tile elements g + (j << 9), j < 8.
template <int OP>
__device__ __forceinline__ void head_levels(uint32_t* planes, uint32_t (&v)[8][kC]) {
  const int g = threadIdx.x;
  reg_levels<OP, 3>(v, 0);
  const int pb = pidx(g);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int q = pb ^ pidx(j << 9);
#pragma unroll
    for (int c = 0; c < kC; ++c) planes[c * kPlane + q] = v[j][c];
  }
  __syncthreads();
}

// Planes, the last R levels (tile bits [zb, zb + R), the first of them level
// lvl of the pass), reduction, stores.
template <int OP, int R, class St>
__device__ __forceinline__ void pass_tail(const uint32_t* planes, int zb, int lvl, St st) {
  constexpr int kGroups = (1 << kMaxTileLog) >> R;
  for (int g = threadIdx.x; g < kGroups; g += blockDim.x) {
    const int base = (g & ((1 << zb) - 1)) | ((g >> zb) << (zb + R));
    const int pb = pidx(base);
    uint32_t v[1 << R][kC];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      const int q = pb ^ pidx(j << zb);
#pragma unroll
      for (int c = 0; c < kC; ++c) v[j][c] = planes[c * kPlane + q];
    }
    reg_levels<OP, R>(v, lvl);
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      Fr w;
#pragma unroll
      for (int c = 0; c < kC; ++c) w.c[c] = tile_final(v[j][c]);
      st(base + (j << zb), pack_fe(w));
    }
  }
}

// Runs the pass on tiles blockIdx.x, blockIdx.x + gridDim.x, ... < n_tiles.
//   fetch(tile, t) -> Raw     the global load of tile element t
//   conv(tile, t, raw) -> Fr  its canonical value
//   st(tile, t, uint4)        the store of the packed result
// Full 4096-element tiles with at least three levels take the register head
// and tail, and the loads of a CTA's next tile are issued right after the
// current tile's head, so they land while its middle and tail stages run.
// A tile is read and written only by the CTA that owns it, so in-place
// passes (src == dst) stay race free.
template <int OP, class Raw, class Fetch, class Conv, class St>
__device__ __forceinline__ void tile_loop(uint32_t* planes, int log_n, int b0, uint32_t n_tiles, Fetch fetch, Conv conv,
                                          St st) {
  const int n = 1 << log_n;
  if (log_n == kMaxTileLog && log_n - b0 >= 3 && blockDim.x == kTileThreads) {
    const int g = threadIdx.x;
    const int rem = 9 - b0;  // level bits [b0, 9) follow the head
    const int rz = rem < 3 ? rem : 3;
    const int rm = rem - rz;
    Raw raw[8];
    uint32_t tile = blockIdx.x;
    if (tile < n_tiles)
#pragma unroll
      for (int j = 0; j < 8; ++j) raw[j] = fetch(tile, g + (j << 9));
    for (; tile < n_tiles; tile += gridDim.x) {
      {
        uint32_t v[8][kC];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const Fr e = conv(tile, g + (j << 9), raw[j]);
#pragma unroll
          for (int c = 0; c < kC; ++c) v[j][c] = e.c[c];
        }
        head_levels<OP>(planes, v);
      }
      const uint32_t next = tile + gridDim.x;
      if (next < n_tiles)
#pragma unroll
        for (int j = 0; j < 8; ++j) raw[j] = fetch(next, g + (j << 9));
      // A radix-4 stage on tile bits 4..5 (b0 = 4) would give a warp's 32
      // groups tile bits 0..3 and 6; bit 6 enters the banks as swizzle
      // column 9, which bits 0..3 also reach (2-way conflicts).  With group
      // bits 4 and 5 swapped the warp covers bits 0..3 and 7 (column 18,
      // bank bit 4): all 32 banks.
      if (b0 == 4 && rm == 2) planar_stage<OP, 2, true>(planes, log_n, 4, 3);
      else planar_levels<OP>(planes, log_n, b0, rm, 3);
      auto st_t = [&](int t, uint4 u) { st(tile, t, u); };
      switch (rz) {
        case 3: pass_tail<OP, 3>(planes, 9 - 3, 3 + rm, st_t); break;
        case 2: pass_tail<OP, 2>(planes, 9 - 2, 3 + rm, st_t); break;
        case 1: pass_tail<OP, 1>(planes, 9 - 1, 3 + rm, st_t); break;
        default:
          for (int t = threadIdx.x; t < n; t += blockDim.x) st(tile, t, planar_get_packed(planes, t));
      }
      __syncthreads();  // the next head overwrites the planes
    }
    return;
  }
  for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) planar_put(planes, t, conv(tile, t, fetch(tile, t)));
    __syncthreads();
    planar_levels<OP>(planes, log_n, b0, log_n - b0);
    for (int t = threadIdx.x; t < n; t += blockDim.x) st(tile, t, planar_get_packed(planes, t));
    __syncthreads();
  }
}


// ---------------------------------------------------------------- element-major tiles
// The transform passes over full 4096-element tiles.  A thread holds whole
// elements (all coefficients, lazily reduced 32-bit values) in registers and
// applies up to three levels to a group of 2^R elements that differ in one
// window of R tile bits; the groups of the next window are formed through
// shared memory.  Shared memory holds the tile element-major: element e's
// coefficients as kUnits 16-byte units, so a thread moves an element with
// kUnits 128-bit accesses.  Unit (e, h) sits at tunit(e, 0) ^ h with
// tunit(e, 0) = (kUnits * e) ^ swz(e), swz XOR-linear in e (F65521: bit 0 =
// e2 ^ e3 ^ e5, bit 1 = e4, bit 2 = e5; KoalaBear: the bits e3..e5).  The
// eight lanes of every 128-bit access phase then hit eight distinct 16-byte
// bank groups for every window the passes use (a simulation of the warps'
// accesses checks [9,12), [0,3), [3,6), [6,9), [2,5), [5,7), [7,9) and the
// windows of the other strided depths).
//
// A pass over tile bits [b0, 12) runs its first window on bits 9..11: a
// thread owns elements g + (j << 9), so consecutive threads load consecutive
// elements.  The remaining bits [b0, 9) are split into windows of at most
// three bits, and the highest window runs last: its groups enumerate tile
// bits 0..4 across the lanes, so the stores are coalesced too.
constexpr int kUnits = kC / 4;
constexpr int kTile = 1 << kMaxTileLog;
__device__ __forceinline__ int tunit(int e) {
  if constexpr (kUnits == 2) return (2 * e) ^ ((((e >> 2) ^ (e >> 3) ^ (e >> 5)) & 1) | ((e >> 3) & 6));
  else return e ^ ((e >> 3) & 7);
}

// Windows of tile bits [b0, 9): at most three bits each, lowest first.
struct Windows {
  int n;
  int b[3], r[3];
};
__device__ __forceinline__ Windows windows_below9(int b0) {
  Windows w{};
  const int span = 9 - b0;
  w.n = (span + 2) / 3;
  int b = b0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int left = 9 - b, parts = w.n - i;
    const int r = parts > 0 ? (left + parts - 1) / parts : 0;
    w.b[i] = b;
    w.r[i] = r;
    b += r;
  }
  return w;
}

// Group g of a window [b, b + R): the elements base + (j << b).
__device__ __forceinline__ int group_base(int g, int b, int R) {
  return (g & ((1 << b) - 1)) | ((g >> b) << (b + R));
}
template <int R>
__device__ __forceinline__ void group_get(const uint4* t, int base, const int (&off)[1 << R], uint32_t (&v)[1 << R][kC]) {
  const int u0 = tunit(base);
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
#pragma unroll
    for (int h = 0; h < kUnits; ++h) {
      const uint4 u = t[(u0 ^ off[j]) ^ h];
      v[j][4 * h] = u.x;
      v[j][4 * h + 1] = u.y;
      v[j][4 * h + 2] = u.z;
      v[j][4 * h + 3] = u.w;
    }
}
template <int R>
__device__ __forceinline__ void group_put(uint4* t, int base, const int (&off)[1 << R], const uint32_t (&v)[1 << R][kC]) {
  const int u0 = tunit(base);
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
#pragma unroll
    for (int h = 0; h < kUnits; ++h)
      t[(u0 ^ off[j]) ^ h] = make_uint4(v[j][4 * h], v[j][4 * h + 1], v[j][4 * h + 2], v[j][4 * h + 3]);
}
template <int R>
__device__ __forceinline__ void window_offsets(int b, int (&off)[1 << R]) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j) off[j] = tunit(j << b);
}

// One window of OP through shared memory (in place: a group is read and
// written by one thread), then a barrier.
template <int OP, int R>
__device__ __forceinline__ void window_stage(uint4* t, int b, int lvl) {
  int off[1 << R];
  window_offsets<R>(b, off);
  for (int g = threadIdx.x; g < (kTile >> R); g += blockDim.x) {
    const int base = group_base(g, b, R);
    uint32_t v[1 << R][kC];
    group_get<R>(t, base, off, v);
    reg_levels<OP, R>(v, lvl);
    group_put<R>(t, base, off, v);
  }
  __syncthreads();
}
template <int OP>
__device__ __forceinline__ void window_stage_r(uint4* t, int b, int r, int lvl) {
  if (r == 3) window_stage<OP, 3>(t, b, lvl);
  else if (r == 2) window_stage<OP, 2>(t, b, lvl);
  else window_stage<OP, 1>(t, b, lvl);
}

// The last window of a pass: OP's levels, reduction to canonical form,
// fin(e, Fr&) on each element (a store to HBM, or the step between two
// transforms), and (PUT) the result back into the tile.
template <int OP, int R, bool PUT, class Fin>
__device__ __forceinline__ void window_last(uint4* t, int b, int lvl, Fin fin) {
  int off[1 << R];
  window_offsets<R>(b, off);
  for (int g = threadIdx.x; g < (kTile >> R); g += blockDim.x) {
    const int base = group_base(g, b, R);
    uint32_t v[1 << R][kC];
    group_get<R>(t, base, off, v);
    reg_levels<OP, R>(v, lvl);
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      Fr w;
#pragma unroll
      for (int c = 0; c < kC; ++c) w.c[c] = tile_final(v[j][c]);
      fin(base + (j << b), w);
#pragma unroll
      for (int c = 0; c < kC; ++c) v[j][c] = w.c[c];
    }
    if (PUT) group_put<R>(t, base, off, v);
  }
}
template <int OP, bool PUT, class Fin>
__device__ __forceinline__ void window_last_r(uint4* t, int b, int r, int lvl, Fin fin) {
  if (r == 3) window_last<OP, 3, PUT>(t, b, lvl, fin);
  else if (r == 2) window_last<OP, 2, PUT>(t, b, lvl, fin);
  else window_last<OP, 1, PUT>(t, b, lvl, fin);
}

// The window where a fused pass changes transforms: OP1's levels, reduction,
// step(e, Fr&) on each canonical element, OP2's first levels, back into the tile.
template <int OP1, int OP2, int R, class Step>
__device__ __forceinline__ void window_mid(uint4* t, int b, int lvl, Step step) {
  int off[1 << R];
  window_offsets<R>(b, off);
  for (int g = threadIdx.x; g < (kTile >> R); g += blockDim.x) {
    const int base = group_base(g, b, R);
    uint32_t v[1 << R][kC];
    group_get<R>(t, base, off, v);
    reg_levels<OP1, R>(v, lvl);
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) {
      Fr x;
#pragma unroll
      for (int c = 0; c < kC; ++c) x.c[c] = tile_final(v[j][c]);
      step(base + (j << b), x);
#pragma unroll
      for (int c = 0; c < kC; ++c) v[j][c] = x.c[c];
    }
    reg_levels<OP2, R>(v, 0);
    group_put<R>(t, base, off, v);
  }
}
template <int OP1, int OP2, class Step>
__device__ __forceinline__ void window_mid_r(uint4* t, int b, int r, int lvl, Step step) {
  if (r == 3) window_mid<OP1, OP2, 3>(t, b, lvl, step);
  else if (r == 2) window_mid<OP1, OP2, 2>(t, b, lvl, step);
  else window_mid<OP1, OP2, 1>(t, b, lvl, step);
}

// A fused pass over full tiles (512 threads): OP1 on tile bits [b0, 12)
// (b0 <= 6), a step on each canonical element, then OP2 on the same bits, in
// one trip through HBM.
//   src(tile, e) -> const void* is the 16-byte global element e of a tile,
//   conv(tile, e, uint4) -> Fr its value;
//   stage(tile) issues the cp.async side loads the step needs (one commit
//   group) into `side`, each thread only to the positions e = g + (j << 9)
//   it owns in the first window;
//   mid(tile, e, Fr&) runs on each canonical element after OP1;
//   st(tile, e, uint4) stores element e (reduced, packed) after OP2.
// `side` (4096 x 16 bytes) also stages the tile's elements: once the step
// has consumed the side loads, each thread copies the next tile's elements
// it owns into its own positions there by cp.async, so they land while OP2
// runs, and reads them back at the next tile's start before stage() reuses
// the positions.  Commit groups: the next tile's elements, then the side
// loads, each waited for in full.
template <int OP1, int OP2, class Src, class Conv, class Stage, class Mid, class St>
__device__ __forceinline__ void tile_pass_v2(uint4* t, uint4* side, int b0, uint32_t n_tiles, Src src, Conv conv, Stage stage,
                                             Mid mid, St st) {
  const int g = threadIdx.x;
  const Windows w = windows_below9(b0);
  int off9[8];
  window_offsets<3>(9, off9);
  uint32_t tile = blockIdx.x;
  if (tile < n_tiles)
#pragma unroll
    for (int j = 0; j < 8; ++j) cp_async16(side + g + (j << 9), src(tile, g + (j << 9)));
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (; tile < n_tiles; tile += gridDim.x) {
    asm volatile("cp.async.wait_all;" ::: "memory");  // this tile's elements (own copies)
    {
      uint32_t v[8][kC];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const Fr e = conv(tile, g + (j << 9), side[g + (j << 9)]);
#pragma unroll
        for (int c = 0; c < kC; ++c) v[j][c] = e.c[c];
      }
      reg_levels<OP1, 3>(v, 0);
      group_put<3>(t, g, off9, v);
    }
    stage(tile);  // into this thread's positions, whose elements it has consumed
    __syncthreads();
    int lvl = 3;
#pragma unroll
    for (int i = 0; i < 2; ++i)
      if (i + 1 < w.n) {
        window_stage_r<OP1>(t, w.b[i], w.r[i], lvl);
        lvl += w.r[i];
      }
    asm volatile("cp.async.wait_all;" ::: "memory");  // the side loads
    __syncthreads();
    const int bl = w.n == 3 ? w.b[2] : (w.n == 2 ? w.b[1] : w.b[0]);
    const int rl = w.n == 3 ? w.r[2] : (w.n == 2 ? w.r[1] : w.r[0]);
    // OP1's last window, the step, and OP2's levels on the same window in
    // registers.
    window_mid_r<OP1, OP2>(t, bl, rl, lvl, [&](int e, Fr& v) { mid(tile, e, v); });
    __syncthreads();  // every step has read the side loads
    const uint32_t next = tile + gridDim.x;
    if (next < n_tiles)
#pragma unroll
      for (int j = 0; j < 8; ++j) cp_async16(side + g + (j << 9), src(next, g + (j << 9)));
    asm volatile("cp.async.commit_group;" ::: "memory");
    int lvl2 = rl;
#pragma unroll
    for (int i = 0; i < 2; ++i)
      if (i + 1 < w.n) {
        window_stage_r<OP2>(t, w.b[i], w.r[i], lvl2);
        lvl2 += w.r[i];
      }
    // OP2's last window: bits 9..11, the elements g + (j << 9), stored.
    {
      uint32_t v[8][kC];
      group_get<3>(t, g, off9, v);
      reg_levels<OP2, 3>(v, lvl2);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        Fr o;
#pragma unroll
        for (int c = 0; c < kC; ++c) o.c[c] = tile_final(v[j][c]);
        st(tile, g + (j << 9), pack_fe(o));
      }
    }
    __syncthreads();  // the next tile's first window overwrites the tile
  }
}

// Pack eight signed weights per element, then Mobius levels [0, levels) in
// tiles of 2^levels elements; write into the message half.  `src_base` is
// the block's first BVA index.
__global__ void __launch_bounds__(kTileThreads, 1) k_pack_mobius_tile(const Wt* __restrict__ bva, uint64_t active,
                                                                     uint64_t src_base, Fe* __restrict__ cw, int logR, int levels,
                                                                     uint32_t n_tiles) {
  extern __shared__ uint32_t planes_s[];
  // kC entries (8 bytes) per element; entries at or past `active` are zero.
  auto fetch = [=](uint32_t tile, int t) {
    const uint64_t g = src_base + uint64_t(kC) * ((uint64_t(tile) << levels) + t);
    if (g + kC <= active) return *reinterpret_cast<const uint2*>(bva + g);
    constexpr int kPer = 4 / int(sizeof(Wt));      // entries per 32-bit word
    constexpr uint32_t kMask = (1u << (8 * sizeof(Wt))) - 1u;
    uint32_t w[2] = {0, 0};
    for (int k = 0; k < kC; ++k)
      if (g + k < active) w[k / kPer] |= (uint32_t(bva[g + k]) & kMask) << (8 * int(sizeof(Wt)) * (k % kPer));
    return make_uint2(w[0], w[1]);
  };
  auto conv = [](uint32_t, int, uint2 raw) { return weights_to_fr(raw); };
  auto st = [=](uint32_t tile, int t, uint4 u) {
    *reinterpret_cast<uint4*>(cw + msg_addr32((tile << levels) + uint32_t(t), logR)) = u;
  };
  tile_loop<kMobius, uint2>(planes_s, levels, 0, n_tiles, fetch, conv, st);
}

// Same, but the packed values come from an element vector (the block-folded
// table), which is left untouched for the sumcheck.
__global__ void __launch_bounds__(kTileThreads, 1) k_copy_mobius_tile(const Fe* __restrict__ src, Fe* __restrict__ cw, int logR,
                                                                     int levels, uint32_t n_tiles) {
  extern __shared__ uint32_t planes_s[];
  auto fetch = [=](uint32_t tile, int t) { return *reinterpret_cast<const uint4*>(src + (size_t(tile) << levels) + t); };
  auto conv = [](uint32_t, int, uint4 raw) { return unpack_fe(raw); };
  auto st = [=](uint32_t tile, int t, uint4 u) {
    *reinterpret_cast<uint4*>(cw + msg_addr32((tile << levels) + uint32_t(t), logR)) = u;
  };
  tile_loop<kMobius, uint4>(planes_s, levels, 0, n_tiles, fetch, conv, st);
}

// WHT levels [0, levels) within tiles (levels <= logR so columns never mix).
// Reads the message (or parity) half at src, with ALPHA multiplies each row
// by alpha[r] first, writes the parity half (src may equal dst).
template <bool ALPHA>
__global__ void __launch_bounds__(ALPHA ? kAlphaTileThreads : kTileThreads, 1)
    k_wht_tile(const Fe* src, Fe* dst, const Fe* __restrict__ alpha, int logR, int levels, uint32_t n_tiles) {
  extern __shared__ uint32_t planes_s[];
  // For a message-half address a = c * 2R + r, a & (R - 1) = r.
  // 32-bit addressing, except with ALPHA, whose extension product leaves no
  // registers for it (that variant spills with it).
  const size_t rmask = (size_t(1) << logR) - 1;
  auto addr = [=](uint32_t tile, int t) -> size_t {
    if constexpr (ALPHA) return msg_addr((size_t(tile) << levels) + t, logR);
    else return msg_addr32((tile << levels) + uint32_t(t), logR);
  };
  auto fetch = [=](uint32_t tile, int t) { return *reinterpret_cast<const uint4*>(src + addr(tile, t)); };
  auto conv = [=](uint32_t tile, int t, uint4 raw) {
    const Fr v = unpack_fe(raw);
    return ALPHA ? mul(v, load(alpha + (addr(tile, t) & rmask))) : v;
  };
  auto st = [=](uint32_t tile, int t, uint4 u) { *reinterpret_cast<uint4*>(dst + addr(tile, t)) = u; };
  tile_loop<kWht, uint4>(planes_s, levels, 0, n_tiles, fetch, conv, st);
}

// Codeword address of element t of tile `tile` of a strided pass: the tile
// owns 2^cb consecutive group bases g0 = tile << cb (64-byte runs in HBM at
// cb = 2, longer above), and tile element t = (j << cb) + c is logical index
// base(g0 + c) + (j << lo), so the pass's k levels act on tile bits [cb, cb + k).
__device__ __forceinline__ uint32_t strided_addr(uint32_t tile, int t, int logR, int lo, int k, int cb) {
  const uint32_t g = (tile << cb) + uint32_t(t & ((1 << cb) - 1));
  return msg_addr32((((g >> lo) << (lo + k)) | (g & ((1u << lo) - 1u))) + (uint32_t(t >> cb) << lo), logR);
}

// Levels [lo, lo + k) over the logical index space of a half: read at `src`
// (cw for the message, cw + R for the parity), written at `dst` (src itself
// for an in-place pass, or the parity half when the first pass of a span
// turns the message into the parity).
template <int OP>
__global__ void __launch_bounds__(kTileThreads, 1) k_butterfly_strided(const Fe* src, Fe* dst, int logR, int lo, int k,
                                                                      int cb, uint32_t n_tiles) {
  extern __shared__ uint32_t planes_s[];
  auto fetch = [=](uint32_t tile, int t) {
    return *reinterpret_cast<const uint4*>(src + strided_addr(tile, t, logR, lo, k, cb));
  };
  auto conv = [](uint32_t, int, uint4 raw) { return unpack_fe(raw); };
  auto st = [=](uint32_t tile, int t, uint4 u) {
    *reinterpret_cast<uint4*>(dst + strided_addr(tile, t, logR, lo, k, cb)) = u;
  };
  tile_loop<OP, uint4>(planes_s, cb + k, cb, n_tiles, fetch, conv, st);
}

// ---------------------------------------------------------------- fused passes
// Two transforms on the same tile bits, with a step on the canonical values
// in between, in one trip through HBM.  The transforms are tensor products of
// 2 x 2 maps on the index bits, so the levels of either one can run in any
// order and levels on different bits commute: a pass may take the message's
// Mobius levels on bits [lo, lo + k) and then the first WHT's levels on the
// same bits, or the first WHT's last levels, the alpha product and the second
// WHT's first levels.

// Registers -> planes: v[j] is tile element base + (j << zb).
template <int R>
__device__ __forceinline__ void regs_to_planes(uint32_t* planes, int base, int zb, const uint32_t (&v)[1 << R][kC]) {
  const int pb = pidx(base);
#pragma unroll
  for (int j = 0; j < (1 << R); ++j) {
    const int q = pb ^ pidx(j << zb);
#pragma unroll
    for (int c = 0; c < kC; ++c) planes[c * kPlane + q] = v[j][c];
  }
}

// Planar levels on tile bits [b0, 6) of a full tile (the levels between a
// register head on bits 9..11 and a register tail on bits 6..8), lvl0 the
// first level's lazy index.  A radix-4 stage on bits 4..5 takes its groups
// with bits 4 and 5 swapped (conflict-free banks, see tile_loop).
template <int OP>
__device__ __forceinline__ void fused_middle(uint32_t* planes, int b0, int lvl0) {
  if (b0 == 4) planar_stage<OP, 2, true>(planes, kMaxTileLog, 4, lvl0);
  else planar_levels<OP>(planes, kMaxTileLog, b0, 6 - b0, lvl0);
}

// Runs OP1 on tile bits [b0, 12) of full 4096-element tiles, then for each
// element mid(tile, t, Fr& v) on its canonical value, then OP2 on the same
// bits, then st(tile, t, uint4).  512 threads, 6 >= b0 >= 0.  OP1: register
// head on bits 9..11, planar levels on [b0, 6), register tail on bits 6..8;
// mid on the tail's registers; OP2: register levels on bits 6..8 right
// there, planar levels on [b0, 6), register tail on bits 9..11 and the
// stores (consecutive threads take consecutive elements, as the loads).
// stage(tile) runs first in each tile (to issue its cp.async side loads,
// which each thread then waits for before the first planar stage's barrier).
// The tile's 16-byte elements (src(tile, t)) arrive by cp.async in a staging
// area of kPrefetchSmem bytes after the planes: thread g copies elements
// g + (j << 9) and reads back only its own copies, so the next tile's copies
// are issued right after the head and land while the rest of the tile runs,
// without holding registers.  Commit groups per tile: the side loads and an
// always-present group closing them, then the next tile's elements.
constexpr size_t kPrefetchSmem = size_t(1) << kMaxTileLog << 4;  // 64 KiB
template <int OP1, int OP2, class Src, class Conv, class Stage, class Mid, class St>
__device__ __forceinline__ void tile_loop_fused(uint32_t* planes, int b0, uint32_t n_tiles, Src src, Conv conv,
                                                Stage stage, Mid mid, St st) {
  const int g = threadIdx.x;
  const int rm = 6 - b0;
  const int tb = (g & 63) | ((g >> 6) << 9);  // the tail group: elements tb + (j << 6)
  uint4* pre = reinterpret_cast<uint4*>(planes + kC * kPlane);
  uint32_t tile = blockIdx.x;
  if (tile < n_tiles)
#pragma unroll
    for (int j = 0; j < 8; ++j) cp_async16(pre + g + (j << 9), src(tile, g + (j << 9)));
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (; tile < n_tiles; tile += gridDim.x) {
    stage(tile);
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");  // this tile's elements (and older groups) have landed
    {
      uint32_t v[8][kC];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const Fr e = conv(tile, g + (j << 9), pre[g + (j << 9)]);
#pragma unroll
        for (int c = 0; c < kC; ++c) v[j][c] = e.c[c];
      }
      head_levels<OP1>(planes, v);
    }
    const uint32_t next = tile + gridDim.x;
    if (next < n_tiles)
#pragma unroll
      for (int j = 0; j < 8; ++j) cp_async16(pre + g + (j << 9), src(next, g + (j << 9)));
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");  // the side loads; the next tile's copies may pend
    if (rm > 0) fused_middle<OP1>(planes, b0, 3);
    else __syncthreads();
    {
      uint32_t v[8][kC];
      const int pb = pidx(tb);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int q = pb ^ pidx(j << 6);
#pragma unroll
        for (int c = 0; c < kC; ++c) v[j][c] = planes[c * kPlane + q];
      }
      reg_levels<OP1, 3>(v, 3 + rm);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        Fr w;
#pragma unroll
        for (int c = 0; c < kC; ++c) w.c[c] = tile_final(v[j][c]);
        mid(tile, tb + (j << 6), w);
#pragma unroll
        for (int c = 0; c < kC; ++c) v[j][c] = w.c[c];
      }
      reg_levels<OP2, 3>(v, 0);
      // The same thread read these positions: no other thread touches them
      // until the barrier below.
      regs_to_planes<3>(planes, tb, 6, v);
    }
    __syncthreads();
    if (rm > 0) fused_middle<OP2>(planes, b0, 3);
    auto st_t = [&](int t, uint4 u) { st(tile, t, u); };
    pass_tail<OP2, 3>(planes, 9, 3 + rm, st_t);
    __syncthreads();  // the next head overwrites the planes
  }
}

// Message half at cw: Mobius levels [lo, lo + k) (the message is final after
// them), stored back; then the first WHT's levels [lo, lo + k) of the same
// values, stored into the parity half at cw + R.  k in [6, 10], cb = 12 - k
// (or 2 at k = 10).
__global__ void __launch_bounds__(kTileThreads, 1) k_mobius_wht_strided(Fe* cw, uint32_t R, int logR, int lo, int k, int cb,
                                                                       uint32_t n_tiles) {
  extern __shared__ uint32_t planes_s[];
  auto src = [=](uint32_t tile, int t) -> const void* { return cw + strided_addr(tile, t, logR, lo, k, cb); };
  auto conv = [](uint32_t, int, uint4 raw) { return unpack_fe(raw); };
  auto stage = [](uint32_t) {};
  auto mid = [=](uint32_t tile, int t, Fr& v) {
    *reinterpret_cast<uint4*>(cw + strided_addr(tile, t, logR, lo, k, cb)) = pack_fe(v);
  };
  auto st = [=](uint32_t tile, int t, uint4 u) {
    *reinterpret_cast<uint4*>(cw + R + strided_addr(tile, t, logR, lo, k, cb)) = u;
  };
  tile_loop_fused<kMobius, kWht>(planes_s, cb, n_tiles, src, conv, stage, mid, st);
}

// The parity tile pass: the first WHT's levels 0..11 of each column (read at
// src, the message half when no strided WHT level came first, else the
// parity half), times alpha[r], the second WHT's levels 0..11, written to the
// parity half at dst.  Each tile's 4096 alphas are staged in shared memory
// (cp.async) while the first WHT runs.
constexpr size_t kAlphaStageSmem = size_t(1) << kMaxTileLog << 4;  // 64 KiB
__global__ void __launch_bounds__(kTileThreads, 1) k_wht_alpha_wht_tile(const Fe* src, Fe* dst, const Fe* __restrict__ alpha,
                                                                       int logR, uint32_t n_tiles) {
  extern __shared__ uint32_t planes_s[];
  uint4* alpha_s = reinterpret_cast<uint4*>(planes_s + kC * kPlane);
  const uint32_t rmask = (1u << logR) - 1u;
  auto addr = [=](uint32_t tile, int t) { return msg_addr32((tile << kMaxTileLog) + uint32_t(t), logR); };
  auto elem = [=](uint32_t tile, int t) -> const void* { return src + addr(tile, t); };
  auto conv = [](uint32_t, int, uint4 raw) { return unpack_fe(raw); };
  auto stage = [=](uint32_t tile) {
    // Tile rows r0 .. r0 + 4095 (R is a multiple of 4096).
    const Fe* a = alpha + ((tile << kMaxTileLog) & rmask);
#pragma unroll
    for (int i = 0; i < (1 << kMaxTileLog) / kTileThreads; ++i) {
      const int e = int(threadIdx.x) + i * kTileThreads;
      cp_async16(alpha_s + e, a + e);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  auto mid = [=](uint32_t, int t, Fr& v) { v = mul(v, unpack_fe(alpha_s[t])); };
  auto st = [=](uint32_t tile, int t, uint4 u) { *reinterpret_cast<uint4*>(dst + addr(tile, t)) = u; };
  // The next tile's elements are staged by cp.async in the alpha area once
  // the step has used it (a register prefetch would spill: measured).
  tile_pass_v2<kWht, kWht>(reinterpret_cast<uint4*>(planes_s), alpha_s, 0, n_tiles, elem, conv, stage, mid, st);
}

// ---------------------------------------------------------------- hashing
// Setup-row leaves (hash_setup_row; qafold_short_setup.rs:655-897): one
// thread per row hashes the framed prefix tail, the framed row index and
// the row's n_cols elements, entry (c, r) at cw[c * n_rows + r].  The message
// is assembled byte by byte; the setup is built once per parameter set,
// outside any proof.
__global__ void k_hash_setup_rows(const Fe* __restrict__ cw, uint64_t n_rows, int n_cols, ::qfd::SetupLeafPrefix pf,
                                  uint4* __restrict__ leaves) {
  const uint64_t row = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (row >= n_rows) return;
  uint32_t h[8], m[16];
#pragma unroll
  for (int i = 0; i < 8; ++i) h[i] = pf.mid[i];
  uint32_t t = pf.t0;
  int fill = 0;
  auto push = [&](uint32_t b) {
    if (fill == 64) {  // a full block is compressed once more input arrives
      t += 64;
      ::qfd::compress(h, m, t, false, pf.one);
      fill = 0;
    }
    const int w = fill >> 2, sh = 8 * (fill & 3);
    m[w] = sh ? (m[w] | (b << sh)) : b;
    ++fill;
  };
  for (uint32_t i = 0; i < pf.n_tail; ++i) push((pf.tail[i >> 2] >> (8 * (i & 3))) & 0xffu);
  // framed "row": u64(3) || "row" || u64(8) || u64(row)
  push(3u);
  for (int i = 0; i < 7; ++i) push(0u);
  push('r');
  push('o');
  push('w');
  push(8u);
  for (int i = 0; i < 7; ++i) push(0u);
  for (int i = 0; i < 8; ++i) push(uint32_t(row >> (8 * i)) & 0xffu);
  for (int c = 0; c < n_cols; ++c) {
    const uint4 u = *reinterpret_cast<const uint4*>(cw + uint64_t(c) * n_rows + row);
    const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int k = 0; k < 16; ++k) push((wd[k >> 2] >> (8 * (k & 3))) & 0xffu);
  }
  t += uint32_t(fill);
  for (int w = (fill + 3) >> 2; w < 16; ++w) m[w] = 0u;
  ::qfd::compress(h, m, t, true, pf.one);
  leaves[2 * row] = make_uint4(h[0], h[1], h[2], h[3]);
  leaves[2 * row + 1] = make_uint4(h[4], h[5], h[6], h[7]);
}

constexpr int kLeafThreads = 64;
constexpr int kRowWords = 128;  // 32 entries x 4 words
constexpr int kRowStride = 129;  // padded: conflict-free per-thread rows

// TAIL = prefix bytes after the 64-byte midstate: 11 for the 75-byte
// base-row prefix, 16 for the 80-byte extension-row prefix.
template <int TAIL>
__global__ void __launch_bounds__(kLeafThreads) k_hash_leaves(const Fe* __restrict__ cw, uint64_t n_rows, int n_cols,
                                                              ::qfd::LeafPrefix pre, uint4* __restrict__ leaves) {
  static_assert(TAIL == 11 || TAIL == 16, "leaf prefix");
  __shared__ uint32_t rows_s[kLeafThreads * kRowStride];
  const uint64_t r = uint64_t(blockIdx.x) * kLeafThreads + threadIdx.x;
  uint32_t* mine = rows_s + threadIdx.x * kRowStride;
  if (r < n_rows) {
    for (int c = 0; c < n_cols; ++c) {
      uint4 u = *reinterpret_cast<const uint4*>(cw + size_t(c) * n_rows + r);
      mine[4 * c] = u.x; mine[4 * c + 1] = u.y; mine[4 * c + 2] = u.z; mine[4 * c + 3] = u.w;
    }
  }
  if (r >= n_rows) return;
  const int nw = 4 * n_cols;  // row words
  auto rw = [&](int q) -> uint32_t { return q < nw ? mine[q] : 0u; };
  uint32_t h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) h[i] = pre.mid[i];
  // Stream after the midstate: TAIL prefix bytes then the row; 64-byte blocks.
  const uint32_t total = 64u + TAIL + uint32_t(nw) * 4u;
  const int nblocks = int((total - 64 + 63) / 64);
  for (int j = 1; j <= nblocks; ++j) {
    uint32_t m[16];
#pragma unroll
    for (int w = 0; w < 16; ++w) {
      const int s = 64 * (j - 1) + 4 * w;
      uint32_t word;
      if (TAIL == 16) {
        word = s < 16 ? pre.tail[w] : rw((s - 16) >> 2);
      } else if (s < 8) {
        word = pre.tail[w];
      } else if (s == 8) {
        word = __byte_perm(pre.tail[2], rw(0), 0x4210);  // pre.tail[2] (3 bytes) | (rw(0) << 24)
      } else {
        const int q = (s - 12) >> 2;
        word = __byte_perm(rw(q), rw(q + 1), 0x4321);  // (rw(q) >> 8) | (rw(q + 1) << 24)
      }
      m[w] = word;
    }
    const bool last = j == nblocks;
    ::qfd::compress(h, m, last ? total : 64u + 64u * uint32_t(j), last, pre.one);
  }
  leaves[2 * r] = make_uint4(h[0], h[1], h[2], h[3]);
  leaves[2 * r + 1] = make_uint4(h[4], h[5], h[6], h[7]);
}

// Inner node = BLAKE2s(50-byte prefix || left || right), 114 bytes.  d holds
// the two children's 16 words; h receives the parent's 8.
__device__ __forceinline__ void inner_hash(const uint32_t (&d)[16], const ::qfd::InnerPrefix& pre, uint32_t (&h)[8]) {
  uint32_t buf[32];
#pragma unroll
  for (int k = 0; k < 12; ++k) buf[k] = pre.w[k];
#pragma unroll
  for (int q = 0; q <= 16; ++q) {
    uint32_t lo = q == 0 ? pre.w[12] : (d[q - 1] >> 16);
    uint32_t hi = q < 16 ? (d[q] << 16) : 0u;
    buf[12 + q] = lo | hi;
  }
#pragma unroll
  for (int k = 29; k < 32; ++k) buf[k] = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) h[k] = ::qfd::kIv[k];
  h[0] ^= 0x01010020u;
  ::qfd::compress(h, buf, 64u, false, pre.one);
  ::qfd::compress(h, buf + 16, 114u, true, pre.one);
}

// Digest offsets (in digests, 2 uint4 each) of the levels a launch reads and
// writes: off[0] the children's level, off[j] the level j above it.
struct TreeLevels {
  uint64_t off[12];
};

// The node at height D above level 0 with index `idx` in its level, from its
// 2^D descendants at level 0; every node it makes is stored in its level.
template <int D>
__device__ __forceinline__ void subtree_hash(uint4* __restrict__ tree, const TreeLevels& lv, uint64_t idx,
                                             const ::qfd::InnerPrefix& pre, uint32_t (&h)[8]) {
  if constexpr (D == 0) {
    const uint4 a = tree[2 * (lv.off[0] + idx)], b = tree[2 * (lv.off[0] + idx) + 1];
    h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w; h[4] = b.x; h[5] = b.y; h[6] = b.z; h[7] = b.w;
  } else {
    uint32_t d[16];
    {
      uint32_t l[8], r[8];
      subtree_hash<D - 1>(tree, lv, 2 * idx, pre, l);
      subtree_hash<D - 1>(tree, lv, 2 * idx + 1, pre, r);
#pragma unroll
      for (int k = 0; k < 8; ++k) { d[k] = l[k]; d[8 + k] = r[k]; }
    }
    inner_hash(d, pre, h);
    tree[2 * (lv.off[D] + idx)] = make_uint4(h[0], h[1], h[2], h[3]);
    tree[2 * (lv.off[D] + idx) + 1] = make_uint4(h[4], h[5], h[6], h[7]);
  }
}

// L inner levels in one launch: thread i hashes the 2^L children [i 2^L,
// (i + 1) 2^L) of level off[0] up to their common ancestor (2^L - 1 node
// hashes, depth first, no barrier), for the n_top nodes of level off[L].
template <int L>
__global__ void k_hash_subtrees(uint4* __restrict__ tree, uint64_t n_top, TreeLevels lv, ::qfd::InnerPrefix pre) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n_top) return;
  uint32_t h[8];
  subtree_hash<L>(tree, lv, i, pre, h);
}

// The top of a tree in one CTA: from the n children at level off[0] (n a
// power of two, n / 2 <= blockDim.x) every level up to the root, one node per
// thread and level, a barrier between levels (the children a level reads are
// the previous level's stores of other threads of this CTA).
__global__ void k_hash_top(uint4* __restrict__ tree, uint64_t n, TreeLevels lv, ::qfd::InnerPrefix pre) {
  int j = 0;
  for (uint64_t parents = n / 2; parents >= 1; parents /= 2, ++j) {
    for (uint64_t i = threadIdx.x; i < parents; i += blockDim.x) {
      const uint4* c = tree + 2 * (lv.off[j] + 2 * i);
      uint32_t d[16];
      const uint4 a = __ldcg(c), b = __ldcg(c + 1), e = __ldcg(c + 2), f = __ldcg(c + 3);
      d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w; d[4] = b.x; d[5] = b.y; d[6] = b.z; d[7] = b.w;
      d[8] = e.x; d[9] = e.y; d[10] = e.z; d[11] = e.w; d[12] = f.x; d[13] = f.y; d[14] = f.z; d[15] = f.w;
      uint32_t h[8];
      inner_hash(d, pre, h);
      tree[2 * (lv.off[j + 1] + i)] = make_uint4(h[0], h[1], h[2], h[3]);
      tree[2 * (lv.off[j + 1] + i) + 1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
    __syncthreads();
  }
}

}  // namespace QFD_NS
