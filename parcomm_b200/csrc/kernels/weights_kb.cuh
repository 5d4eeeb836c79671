// BVA-reading opening kernels for KoalaBear^4 with signed 16-bit payloads:
// TBV lane projections, the packed EO witness, the batch opening's
// equality-table lane projection and the block fold.
//
// A payload (|v| <= 2^15) times a canonical coefficient (< 2^31) is below
// 2^46 in magnitude, so every per-thread and per-warp sum below stays inside
// a signed 64-bit accumulator (the reference keeps u128 raw lanes for the
// same sums, packed_koalabear.rs); each sum is reduced mod p once, and the
// CTA-level totals are kept as canonical residues.
#pragma once
#include <cstdint>

#include "open.cuh"

namespace QFD_NS {

// Four consecutive payloads from entry g (zero at or past `active`); one
// 8-byte load when the four lie inside and g is 4-aligned.
__device__ __forceinline__ uint2 load4(const Wt* __restrict__ bva, uint64_t active, uint64_t g) {
  if (g + 4 <= active && (g & 3) == 0) return *reinterpret_cast<const uint2*>(bva + g);
  uint32_t w[2] = {0, 0};
  for (int j = 0; j < 4; ++j)
    if (g + j < active) w[j >> 1] |= (uint32_t(bva[g + j]) & 0xffffu) << (16 * (j & 1));
  return make_uint2(w[0], w[1]);
}
// c + a * b for a 32-bit signed a and b (a canonical coefficient is below
// 2^31, so it is one): a single widening multiply-add into 64 bits.
__device__ __forceinline__ long long mad_wide(int a, int b, long long c) {
  long long d;
  asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}
// Payload j (0..3) of a load4 word pair.
__device__ __forceinline__ int lane_of(uint2 u, int j) { return int(int16_t(((j < 2 ? u.x : u.y) >> (16 * (j & 1))) & 0xffffu)); }

constexpr int kRowBatch = 2;  // rows whose payload loads a projection thread keeps in flight (measured)

// Lane projections (tbv.rs:288-352): out[tile * lanes + l] = high(tile) *
// sum_r lo[r] * bva[offset + row * lanes + l].  A thread takes min(4, lanes)
// lanes of a row; a tile has at most 4096 rows, so a lane's sum is below
// 2^58 before the single reduction.
__global__ void __launch_bounds__(kTermThreads) k_project_terms(const Wt* __restrict__ bva, uint64_t active,
                                                                const TermTiles* __restrict__ terms, int n_terms,
                                                                uint32_t n_tiles, const Fe* __restrict__ tables,
                                                                int lanes, Fe* __restrict__ out) {
  __shared__ int t_sel;
  __shared__ long long part_s[kTermThreads / 32][64][kC];
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
    long long acc[4][kC];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < kC; ++k) acc[j][k] = 0;
    const Fe* lo = tables + T.lo_off;
    for (int r0 = threadIdx.x / tpr; r0 < nrows; r0 += kRowBatch * rpp) {
      uint2 u[kRowBatch];
#pragma unroll
      for (int q = 0; q < kRowBatch; ++q) {
        const int r = r0 + q * rpp;
        const uint64_t g = T.offset + (row0 + r) * lanes + sub * lpt;
        u[q] = make_uint2(0, 0);
        if (r < nrows) {
          if (lpt == 4) {
            u[q] = load4(bva, active, g);
          } else {
            for (int j = 0; j < lpt; ++j)
              if (g + j < active) (j < 2 ? u[q].x : u[q].y) |= (uint32_t(bva[g + j]) & 0xffffu) << (16 * (j & 1));
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
          const int v = lane_of(u[q], j);
#pragma unroll
          for (int k = 0; k < kC; ++k) acc[j][k] = mad_wide(int(w.c[k]), v, acc[j][k]);
        }
      }
    }
    for (int o = tpr; o < 32; o <<= 1)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < kC; ++k) acc[j][k] += __shfl_xor_sync(0xffffffffu, acc[j][k], o);
    if (lane_id < tpr)
      for (int j = 0; j < lpt; ++j)
#pragma unroll
        for (int k = 0; k < kC; ++k) part_s[warp][lane_id * lpt + j][k] = acc[j][k];
    __syncthreads();
    if (threadIdx.x < lanes) {
      long long s[kC];
#pragma unroll
      for (int k = 0; k < kC; ++k) s[k] = 0;
      for (int w = 0; w < kTermThreads / 32; ++w)
#pragma unroll
        for (int k = 0; k < kC; ++k) s[k] += part_s[w][threadIdx.x][k];
      Fr sum;
#pragma unroll
      for (int k = 0; k < kC; ++k) sum.c[k] = mod_i64(s[k]);
      store(out + size_t(tile) * lanes + threadIdx.x, mul(tile_high(T, tables, i), sum));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- EO
// One full row of L payloads (L a multiple of 8, the row 16-byte aligned):
// 16-byte loads of eight payloads, two accumulator chains (even and odd
// lanes) so consecutive multiply-adds do not wait on each other.
template <int L>
__device__ __forceinline__ void witness_row(const Wt* __restrict__ row, const Fe* pw, long long (&acc)[kC]) {
  long long a2[kC];
#pragma unroll
  for (int k = 0; k < kC; ++k) a2[k] = 0;
#pragma unroll 2
  for (int c = 0; c < L / 8; ++c) {
    const uint4 u = *reinterpret_cast<const uint4*>(row + 8 * c);
    const uint2 lo = make_uint2(u.x, u.y), hi = make_uint2(u.z, u.w);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int v = lane_of(j < 4 ? lo : hi, j & 3);
      const Fr p = load(pw + 8 * c + j);
#pragma unroll
      for (int k = 0; k < kC; ++k) {
        if (j & 1) a2[k] = mad_wide(int(p.c[k]), v, a2[k]);
        else acc[k] = mad_wide(int(p.c[k]), v, acc[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kC; ++k) acc[k] += a2[k];
}

// Packed EO witness (eo.rs:119-132): witness[row] = sum_lane v(row * stride +
// lane) * inv_powers[lane], stride <= 64, so a sum is below 2^52.  Full rows
// of 16 or 64 payloads take the unrolled path; the rest the generic loop.
__global__ void __launch_bounds__(256, 2) k_eo_witness(const Wt* __restrict__ bva, uint64_t active, uint64_t rows,
                                                       int stride, const Fe* __restrict__ inv_powers,
                                                       Fe* __restrict__ witness) {
  __shared__ Fe pw[64];
  if (threadIdx.x < stride) pw[threadIdx.x] = inv_powers[threadIdx.x];
  __syncthreads();
  for (uint64_t row = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; row < rows; row += uint64_t(gridDim.x) * blockDim.x) {
    long long acc[kC];
#pragma unroll
    for (int k = 0; k < kC; ++k) acc[k] = 0;
    const uint64_t g0 = row * stride;
    if (stride == 16 && g0 + 16 <= active) {
      witness_row<16>(bva + g0, pw, acc);
    } else if (stride == 64 && g0 + 64 <= active) {
      witness_row<64>(bva + g0, pw, acc);
    } else if (g0 < active) {
      for (int l0 = 0; l0 < stride; l0 += 4) {
        const int n = stride - l0 < 4 ? stride - l0 : 4;
        const uint2 u = n == 4 ? load4(bva, active, g0 + l0) : make_uint2(0, 0);
        for (int j = 0; j < n; ++j) {
          const uint64_t g = g0 + l0 + j;
          const int v = n == 4 ? lane_of(u, j) : (g < active ? int(bva[g]) : 0);
          const Fr p = load(pw + l0 + j);
#pragma unroll
          for (int k = 0; k < kC; ++k) acc[k] = mad_wide(int(p.c[k]), v, acc[k]);
        }
      }
    }
    Fr w;
#pragma unroll
    for (int k = 0; k < kC; ++k) w.c[k] = mod_i64(acc[k]);
    store(witness + row, w);
  }
}

// ---------------------------------------------------------------- batch opening
// Raw lane sums of up to kEqBlocks consecutive blocks against the equality
// weights (project_lanes_from_fn, packed_batch.rs:25-41):
//   raw[b][j * 4 + k] += sum_i v(b, 4i + j) * weights[i].c[k]
// Blocks go two at a time: a thread keeps both blocks' 16 sums in registers
// over its whole grid-stride range (each weight read once per pair), and the
// CTA reduces once per pair.  A thread handles at most m / (grid x 256)
// elements (below 2^11 for the grids the host launches), so a sum stays below
// 2^57 and a warp sum below 2^62; each warp's sum is reduced to a residue
// before the warps are added, and `raw` receives one atomic add per entry and
// CTA (a sum of residues, far below 2^63).
__global__ void __launch_bounds__(kEqThreads) k_eq_project_blocks(const Wt* __restrict__ bva, uint64_t active,
                                                                 uint64_t block_len, uint64_t first_block, int nb,
                                                                 uint64_t m, const Fe* __restrict__ weights,
                                                                 unsigned long long* __restrict__ raw) {
  __shared__ long long stage_s[kEqThreads / 32][2 * kEqRaw];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int b0 = 0; b0 < nb; b0 += 2) {
    const bool two = b0 + 1 < nb;
    const uint64_t base0 = (first_block + b0) * block_len, base1 = base0 + block_len;
    long long acc[2][kEqRaw];
#pragma unroll
    for (int q = 0; q < kEqRaw; ++q) acc[0][q] = acc[1][q] = 0;
    for (uint64_t i = uint64_t(blockIdx.x) * kEqThreads + threadIdx.x; i < m; i += uint64_t(gridDim.x) * kEqThreads) {
      const uint4 wq = *reinterpret_cast<const uint4*>(weights + i);
      const uint32_t wc[4] = {wq.x, wq.y, wq.z, wq.w};
      const uint2 v0 = load4(bva, active, base0 + 4 * i);
      const uint2 v1 = two ? load4(bva, active, base1 + 4 * i) : make_uint2(0, 0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int a = lane_of(v0, j), b = lane_of(v1, j);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          acc[0][j * 4 + k] = mad_wide(int(wc[k]), a, acc[0][j * 4 + k]);
          acc[1][j * 4 + k] = mad_wide(int(wc[k]), b, acc[1][j * 4 + k]);
        }
      }
    }
    // Reduce-scatter per block: after offset o the lane keeps the half of its
    // entries selected by (lane & o); after o = 2 lane l holds entry l >> 1,
    // and the o = 1 exchange completes the sum in both lanes of the pair.
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int o = 16, n = kEqRaw; o >= 2; o >>= 1, n >>= 1) {
        const bool upper = lane & o;
#pragma unroll
        for (int q = 0; q < n / 2; ++q) {
          const long long send = upper ? acc[h][q] : acc[h][q + n / 2];
          const long long keep = upper ? acc[h][q + n / 2] : acc[h][q];
          acc[h][q] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
      acc[h][0] += __shfl_xor_sync(0xffffffffu, acc[h][0], 1);
      if ((lane & 1) == 0) stage_s[warp][h * kEqRaw + (lane >> 1)] = acc[h][0];
    }
    __syncthreads();
    if (threadIdx.x < (two ? 2 : 1) * kEqRaw) {
      unsigned long long t = 0;
#pragma unroll
      for (int w = 0; w < kEqThreads / 32; ++w) t += mod_i64(stage_s[w][threadIdx.x]);
      atomicAdd(raw + uint64_t(b0) * kEqRaw + threadIdx.x, t % P);
    }
    __syncthreads();
  }
}

// Block fold of the packed payloads (packed_batch.rs:213-236): values[i] =
// sum_b sum_j v(b * block_len + 4i + j) * T[b * 4 + j], T[b * 4 + j] =
// (c^-1)^b * X^j, held in shared memory; with `accumulate` the sum is added
// to values[i].  At most 128 blocks: a sum of 512 products stays below 2^55.
__global__ void k_block_fold(const Wt* __restrict__ bva, uint64_t active, uint64_t block_len, int blocks, uint64_t m,
                             const Fe* __restrict__ T, Fe* __restrict__ values, int accumulate) {
  extern __shared__ uint4 smem_u4[];
  Fe* t_s = reinterpret_cast<Fe*>(smem_u4);
  for (int t = threadIdx.x; t < blocks * kC; t += blockDim.x) t_s[t] = T[t];
  __syncthreads();
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    // Four blocks' loads are issued before their products; even and odd
    // lanes feed two accumulator chains.
    long long acc[2][kC];
#pragma unroll
    for (int k = 0; k < kC; ++k) acc[0][k] = acc[1][k] = 0;
    for (int b = 0; b < blocks && uint64_t(b) * block_len + 4 * i < active; b += 4) {
      uint2 v4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint64_t g = uint64_t(b + q) * block_len + 4 * i;
        v4[q] = (b + q < blocks && g < active) ? load4(bva, active, g) : make_uint2(0, 0);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (b + q >= blocks) break;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int v = lane_of(v4[q], j);
          const Fr t = load(t_s + (b + q) * kC + j);
#pragma unroll
          for (int k = 0; k < kC; ++k) acc[j & 1][k] = mad_wide(int(t.c[k]), v, acc[j & 1][k]);
        }
      }
    }
    Fr o;
#pragma unroll
    for (int k = 0; k < kC; ++k) o.c[k] = mod_i64(acc[0][k] + acc[1][k]);
    store(values + i, accumulate ? add(load(values + i), o) : o);
  }
}

}  // namespace QFD_NS
