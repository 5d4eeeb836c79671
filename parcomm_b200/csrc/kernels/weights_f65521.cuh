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
  for (uint64_t row = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; row < rows; row += uint64_t(gridDim.x) * blockDim.x) {
    int32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const uint64_t g0 = row * stride;
    if (stride == 16 && g0 + 16 <= active) {
      const uint4 raw = *reinterpret_cast<const uint4*>(bva + g0);
      const uint32_t a[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        int32_t lo = 0, hi = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          lo = dp4a_su(a[q], plo[k][q], lo);
          hi = dp4a_su(a[q], phi[k][q], hi);
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

// Raw lane sums of up to kEqBlocks consecutive blocks against the equality
// weights (project_lanes_from_fn, packed_batch.rs:25-41):
//   raw[b][j * 8 + k] += sum_i v(b, 8i + j) * weights[i].c[k]
// A CTA stages a chunk of kEqChunk weights in shared memory and runs every
// block over it, so the table is read from HBM once for all blocks.  A thread
// takes 8 elements per block (one 8-byte load each) into 64 i32 sums; a warp
// reduce-scatter leaves lane l with entries 2l and 2l + 1 (each a sum of 256
// products, |sum| <= 256 * 128 * 65520 < 2^31), and the CTA keeps i64 totals
// per block that reach `raw` with one atomic add per entry at the end.
__global__ void __launch_bounds__(kEqThreads, 2) k_eq_project_blocks(const int8_t* __restrict__ bva, uint64_t active,
                                                                    uint64_t block_len, uint64_t first_block, int nb,
                                                                    uint64_t m, const Fe* __restrict__ weights,
                                                                    unsigned long long* __restrict__ raw) {
  __shared__ uint4 w_s[kEqChunk];
  __shared__ int32_t stage_s[kEqThreads / 32][64];
  __shared__ long long tot_s[kEqBlocks][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = threadIdx.x; t < kEqBlocks * 64; t += kEqThreads) tot_s[t >> 6][t & 63] = 0;
  for (uint64_t c0 = uint64_t(blockIdx.x) * kEqChunk; c0 < m; c0 += uint64_t(gridDim.x) * kEqChunk) {
    __syncthreads();
    for (int e = threadIdx.x; e < kEqChunk; e += kEqThreads)
      w_s[e] = c0 + e < m ? *reinterpret_cast<const uint4*>(weights + c0 + e) : make_uint4(0, 0, 0, 0);
    __syncthreads();
    for (int b = 0; b < nb; ++b) {
      const uint64_t bbase = (first_block + b) * block_len;
      int32_t acc[64];
#pragma unroll
      for (int q = 0; q < 64; ++q) acc[q] = 0;
#pragma unroll 2
      for (int u = 0; u < kEqChunk / kEqThreads; ++u) {
        const int e = threadIdx.x + u * kEqThreads;
        const uint64_t g = bbase + 8 * (c0 + e);
        uint2 v8 = make_uint2(0, 0);
        if (c0 + e < m) {
          if (g + 8 <= active) {
            v8 = *reinterpret_cast<const uint2*>(bva + g);
          } else {
            uint32_t w[2] = {0, 0};
            for (int j = 0; j < 8; ++j)
              if (g + j < active) w[j >> 2] |= uint32_t(uint8_t(bva[g + j])) << (8 * (j & 3));
            v8 = make_uint2(w[0], w[1]);
          }
        }
        const uint4 wq = w_s[e];
        const uint32_t wc[4] = {wq.x, wq.y, wq.z, wq.w};
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int v = int(int8_t(((j < 4 ? v8.x : v8.y) >> (8 * (j & 3))) & 0xffu));
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[j * 8 + k] += v * int32_t((wc[k >> 1] >> (16 * (k & 1))) & 0xffffu);
        }
      }
      // Reduce-scatter over the warp: after offset o the lane keeps the half
      // of its entries selected by (lane & o).
#pragma unroll
      for (int o = 16, n = 64; o >= 1; o >>= 1, n >>= 1) {
        const bool upper = lane & o;
#pragma unroll
        for (int q = 0; q < n / 2; ++q) {
          const int32_t send = upper ? acc[q] : acc[q + n / 2];
          const int32_t keep = upper ? acc[q + n / 2] : acc[q];
          acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
      stage_s[warp][2 * lane] = acc[0];
      stage_s[warp][2 * lane + 1] = acc[1];
      __syncthreads();
      if (threadIdx.x < 64) {
        long long t = 0;
#pragma unroll
        for (int w = 0; w < kEqThreads / 32; ++w) t += stage_s[w][threadIdx.x];
        tot_s[b][threadIdx.x] += t;
      }
      __syncthreads();
    }
  }
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
