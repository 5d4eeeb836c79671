// BVA-reading opening kernels for F65521^8 with signed 8-bit weights: TBV
// lane projections, the packed EO witness, the batch opening's equality-table
// lane projection and the block fold.  Products of 8-bit weights and 16-bit
// coefficients sum exactly in 32-bit registers (dp4a on byte planes where the
// layout allows) and in 64-bit across threads; each sum is reduced mod p once.
#pragma once
#include <cstdint>

#include "open.cuh"

namespace QFD_NS {

// |v| < 2^31: v + 32768 p is in [0, 2^32), then the 2^16 = 15 fold.
__device__ __forceinline__ uint32_t mod_i32(int32_t v) {
  return red32(uint32_t(int64_t(v) + int64_t(P) * 32768));
}
// Four signed 8-bit lanes of a times four unsigned 8-bit lanes of b, plus c.
__device__ __forceinline__ int32_t dp4a_su(uint32_t a, uint32_t b, int32_t c) {
  int32_t d;
  asm("dp4a.s32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
// 4 x 4 byte transpose: out[b] = byte b of x0, x1, x2, x3 (in that order).
__device__ __forceinline__ void transpose4(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, uint32_t (&out)[4]) {
  const uint32_t t0 = __byte_perm(x0, x1, 0x5140), t1 = __byte_perm(x0, x1, 0x7362);
  const uint32_t t2 = __byte_perm(x2, x3, 0x5140), t3 = __byte_perm(x2, x3, 0x7362);
  out[0] = __byte_perm(t0, t2, 0x5410);
  out[1] = __byte_perm(t0, t2, 0x7632);
  out[2] = __byte_perm(t1, t3, 0x5410);
  out[3] = __byte_perm(t1, t3, 0x7632);
}

// Byte planes of the coefficient k of four elements e[0..3]: lo = the low
// bytes, hi = the high bytes, lane i in byte i.
__device__ __forceinline__ void byte_planes(const Fe* e, int k, uint32_t& lo, uint32_t& hi) {
  lo = 0;
  hi = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t c = e[i].c[k];
    lo |= (c & 0xffu) << (8 * i);
    hi |= (c >> 8) << (8 * i);
  }
}

constexpr int kRowBatch = 8;  // rows whose weight loads a projection thread keeps in flight (measured)

// Lane projections (tbv.rs:288-352): out[tile * lanes + l] = high(tile) *
// sum_r lo[r] * bva[offset + row * lanes + l].  A thread takes min(4, lanes)
// lanes of a row (one 32-bit load); products accumulate exactly in i32 per
// thread (a tile has at most 4096 rows, so a thread sums at most 64 rows:
// 64 * 128 * 65520 < 2^30), then in i64 across threads and warps, then
// reduce once.
__global__ void __launch_bounds__(kTermThreads) k_project_terms(const int8_t* __restrict__ bva, uint64_t active,
                                                                const TermTiles* __restrict__ terms, int n_terms,
                                                                uint32_t n_tiles, const Fe* __restrict__ tables,
                                                                int lanes, Fe* __restrict__ out) {
  __shared__ int t_sel;
  __shared__ int64_t part_s[kTermThreads / 32][64][8];
  const uint32_t tile0 = blockIdx.x * kTilesPerCta;
  if (threadIdx.x == 0) t_sel = find_term(terms, n_terms, tile0);
  __syncthreads();
  int ti = t_sel;
  const int lpt = lanes < 4 ? lanes : 4;
  const int tpr = lanes / lpt;
  const int rpp = kTermThreads / tpr;
  const int sub = threadIdx.x % tpr;
  const int warp = threadIdx.x >> 5, lane_id = threadIdx.x & 31;
  for (uint32_t tile = tile0; tile < tile0 + kTilesPerCta && tile < n_tiles; ++tile) {
    while (ti + 1 < n_terms && terms[ti + 1].first_tile <= tile) ++ti;
    const TermTiles T = terms[ti];
    const uint64_t i = tile - T.first_tile + T.tile_skip;
    const uint64_t row0 = i << T.lb;
    const uint64_t span = uint64_t(1) << T.lb, left = T.rows - row0;
    const int nrows = int(left < span ? left : span);
    int32_t acc[4][8];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[j][k] = 0;
    const Fe* lo = tables + T.lo_off;
    // kRowBatch rows per iteration: their loads are issued before any is used.
    for (int r0 = threadIdx.x / tpr; r0 < nrows; r0 += kRowBatch * rpp) {
      uint32_t u[kRowBatch];
#pragma unroll
      for (int q = 0; q < kRowBatch; ++q) {
        const int r = r0 + q * rpp;
        const uint64_t g = T.offset + (row0 + r) * lanes + sub * lpt;
        u[q] = 0;
        if (r < nrows) {
          if (lpt == 4 && g + 4 <= active && (g & 3) == 0) {
            u[q] = *reinterpret_cast<const uint32_t*>(bva + g);
          } else {
            for (int j = 0; j < lpt; ++j)
              if (g + j < active) u[q] |= uint32_t(uint8_t(bva[g + j])) << (8 * j);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < kRowBatch; ++q) {
        const int r = r0 + q * rpp;
        if (r >= nrows) break;
        const Fr w = load(lo + r);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int v = int(int8_t(u[q] >> (8 * j)));
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[j][k] += int32_t(w.c[k]) * v;
        }
      }
    }
    int64_t wide[4][8];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 8; ++k) wide[j][k] = acc[j][k];
    for (int o = tpr; o < 32; o <<= 1)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < 8; ++k) wide[j][k] += __shfl_xor_sync(0xffffffffu, wide[j][k], o);
    if (lane_id < tpr)
      for (int j = 0; j < lpt; ++j)
#pragma unroll
        for (int k = 0; k < 8; ++k) part_s[warp][lane_id * lpt + j][k] = wide[j][k];
    __syncthreads();
    if (threadIdx.x < lanes) {
      int64_t s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int w = 0; w < kTermThreads / 32; ++w)
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] += part_s[w][threadIdx.x][k];
      Fr sum;
#pragma unroll
      for (int k = 0; k < 8; ++k) sum.c[k] = mod_i64(s[k]);
      store(out + size_t(tile) * lanes + threadIdx.x, mul(tile_high(T, tables, i), sum));
    }
    __syncthreads();
  }
}

// Lane projections of terms with 16 lanes (stride 16), in dp4a form: a
// thread takes groups of 4 rows, lanes 8 lh .. 8 lh + 7 and coefficients
// 4 h .. 4 h + 3 (thread 4 g + 2 lh + h).  The 4 rows' weights of a lane and
// the 4 rows' low (high) bytes of a table coefficient transpose into words,
// so each dp4a adds 4 products.  A thread sums at most 16 rows of a tile
// (16 * 128 * 65520 < 2^28), a warp reduce-scatter over the 8 lanes of the
// same (lh, h) stays below 2^31, then i64 across warps and one reduction.
__global__ void __launch_bounds__(kTermThreads) k_project_terms16(const int8_t* __restrict__ bva, uint64_t active,
                                                                  const TermTiles* __restrict__ terms, int n_terms,
                                                                  uint32_t n_tiles, const Fe* __restrict__ tables,
                                                                  Fe* __restrict__ out) {
  __shared__ int t_sel;
  __shared__ int64_t part_s[kTermThreads / 32][16][8];
  const uint32_t tile0 = blockIdx.x * kTilesPerCta;
  if (threadIdx.x == 0) t_sel = find_term(terms, n_terms, tile0);
  __syncthreads();
  int ti = t_sel;
  const int h = threadIdx.x & 1, lh = (threadIdx.x >> 1) & 1, grp = threadIdx.x >> 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kGroups = kTermThreads / 4;
  for (uint32_t tile = tile0; tile < tile0 + kTilesPerCta && tile < n_tiles; ++tile) {
    while (ti + 1 < n_terms && terms[ti + 1].first_tile <= tile) ++ti;
    const TermTiles T = terms[ti];
    const uint64_t i = tile - T.first_tile + T.tile_skip;
    const uint64_t row0 = i << T.lb;
    const uint64_t span = uint64_t(1) << T.lb, left = T.rows - row0;
    const int nrows = int(left < span ? left : span);
    const Fe* lot = tables + T.lo_off;
    int32_t lo[8][4], hi[8][4];
#pragma unroll
    for (int l = 0; l < 8; ++l)
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) lo[l][kk] = hi[l][kk] = 0;
    // Two groups of 4 rows per iteration, all their loads issued first.
    for (int r0 = 4 * grp; r0 < nrows; r0 += 8 * kGroups) {
      uint32_t x[2][8], y[2][8];
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int rr = r0 + q * 4 * kGroups + r;
          const uint64_t g = T.offset + (row0 + rr) * 16 + 8 * lh;
          uint2 u = make_uint2(0, 0), w = make_uint2(0, 0);
          if (rr < nrows) {
            w = reinterpret_cast<const uint2*>(lot + rr)[h];
            if (g + 8 <= active) {
              u = *reinterpret_cast<const uint2*>(bva + g);
            } else {
              uint32_t b[2] = {0, 0};
              for (int y2 = 0; y2 < 8; ++y2)
                if (g + y2 < active) b[y2 >> 2] |= uint32_t(uint8_t(bva[g + y2])) << (8 * (y2 & 3));
              u = make_uint2(b[0], b[1]);
            }
          }
          x[q][2 * r] = u.x;
          x[q][2 * r + 1] = u.y;
          y[q][2 * r] = w.x;
          y[q][2 * r + 1] = w.y;
        }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        uint32_t va[4], vb[4], pa[4], pb[4];
        transpose4(x[q][0], x[q][2], x[q][4], x[q][6], va);  // lanes 8 lh + 0..3
        transpose4(x[q][1], x[q][3], x[q][5], x[q][7], vb);  // lanes 8 lh + 4..7
        transpose4(y[q][0], y[q][2], y[q][4], y[q][6], pa);  // {lo, hi} of coefficients 4h, 4h + 1
        transpose4(y[q][1], y[q][3], y[q][5], y[q][7], pb);  // {lo, hi} of coefficients 4h + 2, 4h + 3
        const uint32_t plo[4] = {pa[0], pa[2], pb[0], pb[2]}, phi[4] = {pa[1], pa[3], pb[1], pb[3]};
#pragma unroll
        for (int l = 0; l < 8; ++l) {
          const uint32_t v = l < 4 ? va[l] : vb[l - 4];
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            lo[l][kk] = dp4a_su(v, plo[kk], lo[l][kk]);
            hi[l][kk] = dp4a_su(v, phi[kk], hi[l][kk]);
          }
        }
      }
    }
    int32_t acc[32];
#pragma unroll
    for (int f = 0; f < 32; ++f) acc[f] = lo[f >> 2][f & 3] + 256 * hi[f >> 2][f & 3];
    // Reduce-scatter over the 8 lanes with the same (lh, h): the lane keeps
    // entries (lane & 28) .. + 3, i.e. lane 8 lh + ((lane >> 2) & 7),
    // coefficients 4 h .. 4 h + 3.
#pragma unroll
    for (int o = 16, n = 32; o >= 4; o >>= 1, n >>= 1) {
      const bool upper = lane & o;
#pragma unroll
      for (int qq = 0; qq < n / 2; ++qq) {
        const int32_t send = upper ? acc[qq] : acc[qq + n / 2];
        const int32_t keep = upper ? acc[qq + n / 2] : acc[qq];
        acc[qq] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) part_s[warp][8 * lh + ((lane >> 2) & 7)][4 * h + qq] = acc[qq];
    __syncthreads();
    if (threadIdx.x < 16) {
      int64_t sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int w = 0; w < kTermThreads / 32; ++w)
#pragma unroll
        for (int k = 0; k < 8; ++k) sum[k] += part_s[w][threadIdx.x][k];
      Fr v;
#pragma unroll
      for (int k = 0; k < 8; ++k) v.c[k] = mod_i64(sum[k]);
      store(out + size_t(tile) * 16 + threadIdx.x, mul(tile_high(T, tables, i), v));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- EO
// witness[row] = sum_lane v[row * stride + lane] * inv^lane (eo.rs:119-132).
// Packed EO witness (eo.rs:119-132): witness[row] = sum_lane v(row * stride +
// lane) * inv_powers[lane].  For stride 16 a row is one 16-byte load and each
// coefficient two chains of four dp4a (signed weights against the low and
// high bytes of the powers, held in registers); |sum| < 16 * 128 * 65520.
__global__ void k_eo_witness(const int8_t* __restrict__ bva, uint64_t active, uint64_t rows, int stride,
                             const Fe* __restrict__ inv_powers, Fe* __restrict__ witness) {
  __shared__ Fe pw[64];
  if (threadIdx.x < stride) pw[threadIdx.x] = inv_powers[threadIdx.x];
  __syncthreads();
  uint32_t plo[8][4], phi[8][4];
  if (stride == 16) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int q = 0; q < 4; ++q) byte_planes(pw + 4 * q, k, plo[k][q], phi[k][q]);
  }
  // kWitRows rows per thread and iteration, their loads issued first, so that
  // enough 16-byte loads are in flight to keep HBM busy.
  constexpr int kWitRows = 4;
  const uint64_t nthr = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t row0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; row0 < rows; row0 += kWitRows * nthr) {
    uint4 raw[kWitRows];
#pragma unroll
    for (int q = 0; q < kWitRows; ++q) {
      const uint64_t row = row0 + q * nthr;
      raw[q] = (stride == 16 && row < rows && row * 16 + 16 <= active)
                   ? *reinterpret_cast<const uint4*>(bva + row * 16)
                   : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int q = 0; q < kWitRows; ++q) {
      const uint64_t row = row0 + q * nthr;
      if (row >= rows) break;
      int32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      const uint64_t g0 = row * stride;
      if (stride == 16 && g0 + 16 <= active) {
        const uint32_t a[4] = {raw[q].x, raw[q].y, raw[q].z, raw[q].w};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          int32_t lo = 0, hi = 0;
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            lo = dp4a_su(a[c], plo[k][c], lo);
            hi = dp4a_su(a[c], phi[k][c], hi);
          }
          acc[k] = lo + hi * 256;
        }
      } else if (g0 < active) {
        for (int lane = 0; lane < stride; ++lane) {
          const uint64_t g = g0 + lane;
          const int v = g < active ? int(bva[g]) : 0;
          const Fr p = load(pw + lane);
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[k] += int32_t(p.c[k]) * v;
        }
      }
      Fr w;
#pragma unroll
      for (int k = 0; k < 8; ++k) w.c[k] = mod_i32(acc[k]);
      store(witness + row, w);
    }
  }
}


// Raw lane sums of up to kEqBlocks consecutive blocks against the equality
// weights (project_lanes_from_fn, packed_batch.rs:25-41):
//   raw[b][j * 8 + k] += sum_i v(b, 8i + j) * weights[i].c[k]
// in dp4a form: four consecutive elements form a quad; the weights of a quad
// transpose (byte permutes) into one word per lane j holding its 4 entries,
// and the table's coefficient k of the quad into a low-byte and a high-byte
// plane, so one dp4a adds 4 products of a (j, k, byte) entry.  A CTA stages
// a chunk of kEqChunk table entries as byte planes in shared memory (read
// from HBM once for all blocks).  Thread 2q + h takes quad q's lanes j = 0..7
// and coefficients 4h..4h+3.  Per chunk and block a warp covers 256
// elements; a warp reduce-scatter over the 16 lanes of a coefficient half
// leaves each lane two entries (|sum| <= 256 * 128 * 65520 < 2^31), and the
// CTA keeps i64 totals per block that reach `raw` with one atomic add per
// entry at the end.
constexpr size_t kEqWeightSmem = 2 * (kEqChunk / 2) * 16;  // the weight double buffer of k_eq_project_blocks

// 16 bytes of weights from global to shared memory, asynchronously; bytes at
// or past `avail` (0..16) are zero-filled (and not read).
__device__ __forceinline__ void cp_async16_zfill(void* smem, const void* gmem, uint32_t avail) {
  const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(avail) : "memory");
}

__global__ void __launch_bounds__(kEqThreads, 2) k_eq_project_blocks(const int8_t* __restrict__ bva, uint64_t active,
                                                                    uint64_t block_len, uint64_t first_block, int nb,
                                                                    uint64_t m, const Fe* __restrict__ weights,
                                                                    unsigned long long* __restrict__ raw) {
  constexpr int kQuads = kEqChunk / 4;
  // planes_s[q][g]: g = 0 low planes of k 0..3, 1 high planes of k 0..3, 2 and 3 the same for k 4..7.
  __shared__ uint4 planes_s[kQuads][4];
  // The chunk's weights of the block being summed and of the next one
  // (cp.async double buffer, kEqWeightSmem bytes of dynamic shared memory):
  // element e's 8 lanes at bytes 8e .. 8e + 7 of a buffer.
  extern __shared__ uint4 eq_dyn_s[];
  uint4 (*wts_s)[kEqChunk / 2] = reinterpret_cast<uint4 (*)[kEqChunk / 2]>(eq_dyn_s);
  __shared__ int32_t stage_s[kEqThreads / 32][64];
  __shared__ long long tot_s[kEqBlocks][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, h = threadIdx.x & 1;
  for (int t = threadIdx.x; t < kEqBlocks * 64; t += kEqThreads) tot_s[t >> 6][t & 63] = 0;
  // Issues the copies of block b's chunk into wts_s[buf].
  auto stage_block = [&](uint64_t c0, int b, int buf) {
    const uint64_t bbase = (first_block + b) * block_len;
    for (int u = threadIdx.x; u < kEqChunk / 2; u += kEqThreads) {
      const uint64_t i = c0 + 2 * uint64_t(u);  // the unit's first element
      const uint64_t g = bbase + 8 * i;
      uint32_t avail = 0;
      if (i < m && g < active) avail = uint32_t(active - g < 16 ? active - g : 16);
      if (i + 1 >= m && avail > 8) avail = 8;  // the second element is past the packed length
      cp_async16_zfill(&wts_s[buf][u], avail ? static_cast<const void*>(bva + g) : static_cast<const void*>(bva), avail);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  for (uint64_t c0 = uint64_t(blockIdx.x) * kEqChunk; c0 < m; c0 += uint64_t(gridDim.x) * kEqChunk) {
    __syncthreads();
    if (nb > 0) stage_block(c0, 0, 0);
    for (int q = threadIdx.x; q < kQuads; q += kEqThreads) {
      uint4 e[4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
        e[r] = c0 + 4 * q + r < m ? *reinterpret_cast<const uint4*>(weights + c0 + 4 * q + r) : make_uint4(0, 0, 0, 0);
      // Word w of the elements holds coefficients 2w (bytes 0, 1) and 2w + 1 (bytes 2, 3).
      uint32_t pl[4][4];
      transpose4(e[0].x, e[1].x, e[2].x, e[3].x, pl[0]);
      transpose4(e[0].y, e[1].y, e[2].y, e[3].y, pl[1]);
      transpose4(e[0].z, e[1].z, e[2].z, e[3].z, pl[2]);
      transpose4(e[0].w, e[1].w, e[2].w, e[3].w, pl[3]);
      // Group g of quad q sits in slot g ^ ((q >> 1) & 1): a warp phase of 4
      // quads x 2 coefficient halves then reads 8 distinct bank groups.
      const int sw = (q >> 1) & 1;
      planes_s[q][0 ^ sw] = make_uint4(pl[0][0], pl[0][2], pl[1][0], pl[1][2]);
      planes_s[q][1 ^ sw] = make_uint4(pl[0][1], pl[0][3], pl[1][1], pl[1][3]);
      planes_s[q][2 ^ sw] = make_uint4(pl[2][0], pl[2][2], pl[3][0], pl[3][2]);
      planes_s[q][3 ^ sw] = make_uint4(pl[2][1], pl[2][3], pl[3][1], pl[3][3]);
    }
    for (int b = 0; b < nb; ++b) {
      if (b + 1 < nb) {
        stage_block(c0, b + 1, (b + 1) & 1);
        asm volatile("cp.async.wait_group 1;" ::: "memory");
      } else {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
      }
      __syncthreads();  // block b's weights (and, at b = 0, the planes) are in shared memory
      const uint4* wb = wts_s[b & 1];
      int32_t lo[8][4], hi[8][4];
#pragma unroll
      for (int jj = 0; jj < 8; ++jj)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) lo[jj][kk] = hi[jj][kk] = 0;
#pragma unroll 2
      for (int u = 0; u < kQuads / (kEqThreads / 2); ++u) {
        const int q = (threadIdx.x >> 1) + u * (kEqThreads / 2);
        const uint4 a = wb[2 * q], bq = wb[2 * q + 1];
        // vj[jj]: lane jj of the quad's 4 elements (element r's lanes are words 2r, 2r + 1).
        uint32_t v_lo[4], v_hi[4];
        transpose4(a.x, a.z, bq.x, bq.z, v_lo);
        transpose4(a.y, a.w, bq.y, bq.w, v_hi);
        const int sw = (q >> 1) & 1;
        const uint4 pl = planes_s[q][(2 * h) ^ sw], ph = planes_s[q][(2 * h + 1) ^ sw];
        const uint32_t plo[4] = {pl.x, pl.y, pl.z, pl.w}, phi[4] = {ph.x, ph.y, ph.z, ph.w};
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const uint32_t v = jj < 4 ? v_lo[jj] : v_hi[jj - 4];
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            lo[jj][kk] = dp4a_su(v, plo[kk], lo[jj][kk]);
            hi[jj][kk] = dp4a_su(v, phi[kk], hi[jj][kk]);
          }
        }
      }
      int32_t acc[32];
#pragma unroll
      for (int f = 0; f < 32; ++f) acc[f] = lo[f >> 2][f & 3] + 256 * hi[f >> 2][f & 3];
      // Reduce-scatter over the 16 lanes of this coefficient half: after
      // offset o the lane keeps the half of its entries selected by (lane & o);
      // it ends with entries (lane & 30) and (lane & 30) + 1.
#pragma unroll
      for (int o = 16, n = 32; o >= 2; o >>= 1, n >>= 1) {
        const bool upper = lane & o;
#pragma unroll
        for (int qq = 0; qq < n / 2; ++qq) {
          const int32_t send = upper ? acc[qq] : acc[qq + n / 2];
          const int32_t keep = upper ? acc[qq + n / 2] : acc[qq];
          acc[qq] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
#pragma unroll
      for (int qq = 0; qq < 2; ++qq) {
        const int f = (lane & 30) + qq;  // entry f: lane j = f / 4, coefficient 4h + f % 4
        stage_s[warp][(f >> 2) * 8 + 4 * h + (f & 3)] = acc[qq];
      }
      __syncthreads();  // stage_s complete; every thread is done reading wts_s[b & 1]
      if (threadIdx.x < 64) {
        long long t = 0;
#pragma unroll
        for (int w = 0; w < kEqThreads / 32; ++w) t += stage_s[w][threadIdx.x];
        tot_s[b][threadIdx.x] += t;
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * 64; t += kEqThreads)
    atomicAdd(raw + t, (unsigned long long)tot_s[t >> 6][t & 63]);  // two's complement sum
}

// Block fold of the packed weights (packed_batch.rs:213-236):
// values[i] = sum_b sum_j v(b * block_len + 8i + j) * T[b * 8 + j], T[b * 8 + j] =
// (c^-1)^b * X^j; with `accumulate` the sum is added to values[i] (blocks
// folded one launch at a time).  Each block's T rows are held as byte planes
// in shared memory; a block contributes two dp4a per byte plane and
// coefficient.  Sums of 8 blocks stay below 8 * 8 * 128 * 65520 < 2^31 and
// move to i64 totals.
__global__ void k_block_fold(const int8_t* __restrict__ bva, uint64_t active, uint64_t block_len, int blocks, uint64_t m,
                             const Fe* __restrict__ T, Fe* __restrict__ values, int accumulate) {
  extern __shared__ uint4 smem_u4[];
  // planes[b][k] = {lo(j 0..3), lo(j 4..7), hi(j 0..3), hi(j 4..7)}
  uint4* planes = smem_u4;
  for (int t = threadIdx.x; t < blocks * 8; t += blockDim.x) {
    const int b = t >> 3, k = t & 7;
    uint4 pl;
    byte_planes(T + b * 8, k, pl.x, pl.z);
    byte_planes(T + b * 8 + 4, k, pl.y, pl.w);
    planes[t] = pl;
  }
  __syncthreads();
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    int32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (blocks <= 8) {
      // Up to 8 blocks: every block's 8 weights are loaded before any is used.
      uint2 v8[8];
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const uint64_t g = uint64_t(b) * block_len + 8 * i;
        v8[b] = make_uint2(0, 0);
        if (b < blocks && g + 8 <= active) {
          v8[b] = *reinterpret_cast<const uint2*>(bva + g);
        } else if (b < blocks && g < active) {
          uint32_t w[2] = {0, 0};
          for (int j = 0; j < 8; ++j)
            if (g + j < active) w[j >> 2] |= uint32_t(uint8_t(bva[g + j])) << (8 * (j & 3));
          v8[b] = make_uint2(w[0], w[1]);
        }
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        if (b >= blocks) break;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const uint4 pl = planes[b * 8 + k];
          const int32_t lo = dp4a_su(v8[b].y, pl.y, dp4a_su(v8[b].x, pl.x, 0));
          const int32_t hi = dp4a_su(v8[b].y, pl.w, dp4a_su(v8[b].x, pl.z, 0));
          acc[k] += lo + hi * 256;
        }
      }
      Fr o;
#pragma unroll
      for (int k = 0; k < 8; ++k) o.c[k] = mod_i32(acc[k]);
      store(values + i, accumulate ? add(load(values + i), o) : o);
      continue;
    }
    for (int b = 0; b < blocks; ++b) {
      if (b && (b & 7) == 0)
#pragma unroll
        for (int k = 0; k < 8; ++k) { tot[k] += acc[k]; acc[k] = 0; }
      const uint64_t g = uint64_t(b) * block_len + 8 * i;
      if (g >= active) break;  // later blocks start even later
      uint2 v8;
      if (g + 8 <= active) {
        v8 = *reinterpret_cast<const uint2*>(bva + g);
      } else {
        uint32_t w[2] = {0, 0};
        for (int j = 0; j < 8; ++j)
          if (g + j < active) w[j >> 2] |= uint32_t(uint8_t(bva[g + j])) << (8 * (j & 3));
        v8 = make_uint2(w[0], w[1]);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint4 pl = planes[b * 8 + k];
        const int32_t lo = dp4a_su(v8.y, pl.y, dp4a_su(v8.x, pl.x, 0));
        const int32_t hi = dp4a_su(v8.y, pl.w, dp4a_su(v8.x, pl.z, 0));
        acc[k] += lo + hi * 256;
      }
    }
    Fr o;
#pragma unroll
    for (int k = 0; k < 8; ++k) o.c[k] = blocks > 8 ? mod_i64(tot[k] + acc[k]) : mod_i32(acc[k]);
    store(values + i, accumulate ? add(load(values + i), o) : o);
  }
}

}  // namespace QFD_NS
