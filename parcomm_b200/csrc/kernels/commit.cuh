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
#include "../device/f65521_dev.cuh"
#include "../device/hash_prefix.h"

namespace qfd {

__device__ __forceinline__ size_t msg_addr(size_t i, int logR) {
  return ((i >> logR) << (logR + 1)) | (i & ((size_t(1) << logR) - 1));
}

enum ButterflyOp { kMobius = 0, kWht = 1 };

template <int OP>
__device__ __forceinline__ void butterfly(Fe* lo, Fe* hi) {
  Fr a = load(lo), b = load(hi);
  if (OP == kMobius) {
    store(hi, sub(b, a));
  } else {
    store(lo, add(a, b));
    store(hi, sub(a, b));
  }
}

// In-shared-memory butterflies over `levels` low levels of a tile of 2^levels
// consecutive elements.
template <int OP>
__device__ __forceinline__ void tile_levels(Fe* tile, int levels) {
  const int n = 1 << levels;
  for (int l = 0; l < levels; ++l) {
    const int half = 1 << l;
    for (int p = threadIdx.x; p < n / 2; p += blockDim.x) {
      int lo = ((p >> l) << (l + 1)) | (p & (half - 1));
      butterfly<OP>(tile + lo, tile + lo + half);
    }
    __syncthreads();
  }
}

// Pack eight signed weights per element, then Mobius levels [0, levels) in a
// tile; write into the message half.  `src_base` is the block's first BVA index.
__global__ void k_pack_mobius_tile(const int8_t* __restrict__ bva, uint64_t active, uint64_t src_base,
                                   Fe* __restrict__ cw, int logR, int levels) {
  extern __shared__ uint4 smem_u4[];
  Fe* tile = reinterpret_cast<Fe*>(smem_u4);
  const int n = 1 << levels;
  const size_t first = size_t(blockIdx.x) << levels;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const uint64_t g = src_base + 8ull * (first + e);
    int8_t v[8];
    if (g + 8 <= active) {
      uint2 raw = *reinterpret_cast<const uint2*>(bva + g);
      const int8_t* b = reinterpret_cast<const int8_t*>(&raw);
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = b[k];
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = (g + k < active) ? bva[g + k] : int8_t(0);
    }
    Fr r;
#pragma unroll
    for (int k = 0; k < 8; ++k) r.c[k] = small(v[k]);
    store(tile + e, r);
  }
  __syncthreads();
  tile_levels<kMobius>(tile, levels);
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const size_t i = first + e;
    *reinterpret_cast<uint4*>(cw + msg_addr(i, logR)) = *reinterpret_cast<const uint4*>(tile + e);
  }
}

// Same as above but the packed values come from an element vector (the
// block-folded table); the source is also left untouched for the sumcheck.
__global__ void k_copy_mobius_tile(const Fe* __restrict__ src, Fe* __restrict__ cw, int logR, int levels) {
  extern __shared__ uint4 smem_u4[];
  Fe* tile = reinterpret_cast<Fe*>(smem_u4);
  const int n = 1 << levels;
  const size_t first = size_t(blockIdx.x) << levels;
  for (int e = threadIdx.x; e < n; e += blockDim.x)
    *reinterpret_cast<uint4*>(tile + e) = *reinterpret_cast<const uint4*>(src + first + e);
  __syncthreads();
  tile_levels<kMobius>(tile, levels);
  for (int e = threadIdx.x; e < n; e += blockDim.x)
    *reinterpret_cast<uint4*>(cw + msg_addr(first + e, logR)) = *reinterpret_cast<const uint4*>(tile + e);
}

// WHT levels [0, levels) within a tile (levels <= logR so columns never mix).
// Reads the message (or parity) half at src, optionally multiplies each row by
// alpha[r] first, writes the parity half.
__global__ void k_wht_tile(const Fe* src, Fe* dst, const Fe* __restrict__ alpha, int logR,
                           int levels) {
  extern __shared__ uint4 smem_u4[];
  Fe* tile = reinterpret_cast<Fe*>(smem_u4);
  const int n = 1 << levels;
  const size_t first = size_t(blockIdx.x) << levels;
  const size_t rmask = (size_t(1) << logR) - 1;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const size_t i = first + e;
    Fr v = load(src + msg_addr(i, logR));
    if (alpha) v = mul(v, load(alpha + (i & rmask)));
    store(tile + e, v);
  }
  __syncthreads();
  tile_levels<kWht>(tile, levels);
  for (int e = threadIdx.x; e < n; e += blockDim.x)
    *reinterpret_cast<uint4*>(dst + msg_addr(first + e, logR)) = *reinterpret_cast<const uint4*>(tile + e);
}

// Levels [lo, lo + k) over the logical index space of m elements, on the half
// starting at `base` (cw for the message, cw + R for the parity).  Each CTA
// owns 8 consecutive group bases (one 128-byte segment per row of the tile).
template <int OP>
__global__ void k_butterfly_strided(Fe* __restrict__ base, int logR, int lo, int k) {
  extern __shared__ uint4 smem_u4[];
  Fe* tile = reinterpret_cast<Fe*>(smem_u4);
  const int rows = 1 << k;
  const size_t g0 = size_t(blockIdx.x) * 8;
  const size_t low_mask = (size_t(1) << lo) - 1;
  for (int t = threadIdx.x; t < rows * 8; t += blockDim.x) {
    const int c8 = t & 7, j = t >> 3;
    const size_t g = g0 + c8;
    const size_t i = (((g >> lo) << (lo + k)) | (g & low_mask)) + (size_t(j) << lo);
    *reinterpret_cast<uint4*>(tile + t) = *reinterpret_cast<const uint4*>(base + msg_addr(i, logR));
  }
  __syncthreads();
  for (int l = 0; l < k; ++l) {
    const int half = 1 << l;
    for (int q = threadIdx.x; q < rows * 4; q += blockDim.x) {
      const int c8 = q & 7, pj = q >> 3;
      const int jlo = ((pj >> l) << (l + 1)) | (pj & (half - 1));
      butterfly<OP>(tile + jlo * 8 + c8, tile + (jlo + half) * 8 + c8);
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < rows * 8; t += blockDim.x) {
    const int c8 = t & 7, j = t >> 3;
    const size_t g = g0 + c8;
    const size_t i = (((g >> lo) << (lo + k)) | (g & low_mask)) + (size_t(j) << lo);
    *reinterpret_cast<uint4*>(base + msg_addr(i, logR)) = *reinterpret_cast<const uint4*>(tile + t);
  }
}

// ---------------------------------------------------------------- hashing
constexpr int kLeafThreads = 64;
constexpr int kRowWords = 128;  // 32 entries x 4 words
constexpr int kRowStride = 129;  // padded: conflict-free per-thread rows

// TAIL = prefix bytes after the 64-byte midstate: 11 for the 75-byte
// base-row prefix, 16 for the 80-byte extension-row prefix.
template <int TAIL>
__global__ void __launch_bounds__(kLeafThreads) k_hash_leaves(const Fe* __restrict__ cw, uint64_t n_rows, int n_cols,
                                                              LeafPrefix pre, uint4* __restrict__ leaves) {
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
        word = pre.tail[2] | (rw(0) << 24);
      } else {
        const int q = (s - 12) >> 2;
        word = (rw(q) >> 8) | (rw(q + 1) << 24);
      }
      m[w] = word;
    }
    const bool last = j == nblocks;
    compress(h, m, last ? total : 64u + 64u * uint32_t(j), last);
  }
  leaves[2 * r] = make_uint4(h[0], h[1], h[2], h[3]);
  leaves[2 * r + 1] = make_uint4(h[4], h[5], h[6], h[7]);
}

// Inner node = BLAKE2s(50-byte prefix || left || right), 114 bytes.
__global__ void k_hash_inner(const uint4* __restrict__ children, uint64_t n_parents, InnerPrefix pre, uint4* __restrict__ parents) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n_parents) return;
  uint32_t d[16];
  uint4 a = children[4 * i], b = children[4 * i + 1], c = children[4 * i + 2], e = children[4 * i + 3];
  d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w; d[4] = b.x; d[5] = b.y; d[6] = b.z; d[7] = b.w;
  d[8] = c.x; d[9] = c.y; d[10] = c.z; d[11] = c.w; d[12] = e.x; d[13] = e.y; d[14] = e.z; d[15] = e.w;
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
  uint32_t h[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) h[k] = kIv[k];
  h[0] ^= 0x01010020u;
  compress(h, buf, 64u, false);
  compress(h, buf + 16, 114u, true);
  parents[2 * i] = make_uint4(h[0], h[1], h[2], h[3]);
  parents[2 * i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
}

}  // namespace qfd
