// Exact integer-limb tensor-core forms of three F65521^8 weight passes: the
// packed EO witness (eo.rs:119-132), the block fold (packed_batch.rs:
// 213-236) and the batch opening's equality-table lane sums (packed_batch.rs:
// 25-41).  Each contracts signed 8-bit weights against a table of extension
// elements.  Each table coefficient (canonical, < 2^16) splits into its two
// bytes, which are exactly the 16 bytes of the element's storage (byte 2k =
// low byte of coefficient k, byte 2k + 1 = its high byte).  One
// mma.sync.m16n8k{16,32} with s8 weights (A) and u8 limbs (B) then sums
// weight x limb products exactly in s32, and coefficient k of an output row
// is limb_sum(2k) + 256 * limb_sum(2k + 1), reduced mod p once.
//
// Fragment layouts (mma.m16n8k16 / m16n8k32, 8-bit A and B): lane = 4g + t;
// a 32-bit A register holds the four consecutive K entries 4t..4t+3 (plus 16
// for the second half of k32) of row g or g + 8; a B register holds K
// entries 4t..4t+3 of column g; the s32 accumulators c0, c1 are row g,
// columns 2t, 2t + 1, and c2, c3 row g + 8.  With the limbs of an element's
// coefficients 0..3 in the first 8-column tile and those of 4..7 in the
// second, a lane's (c0, c1) is the (low, high) limb pair of coefficient t
// (first tile) or t + 4 (second tile).
#pragma once
#include <cstdint>

#include "weights_f65521.cuh"

namespace QFD_NS {

__device__ __forceinline__ void mma_s8u8_k16(int32_t (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
  asm("mma.sync.aligned.m16n8k16.row.col.s32.s8.u8.s32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a0), "r"(a1), "r"(b0));
}
__device__ __forceinline__ void mma_s8u8_k32(int32_t (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k32.row.col.s32.s8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Byte (limb) l of an extension element in storage.
__device__ __forceinline__ uint32_t fe_limb(const Fe* e, int l) {
  const uint32_t w = reinterpret_cast<const uint32_t*>(e)[l >> 2];
  return (w >> (8 * (l & 3))) & 0xffu;
}

// The 32-bit word of weights at BVA index g (a multiple of 4), zero at or
// past `active`.
__device__ __forceinline__ uint32_t weight_word(const int8_t* __restrict__ bva, uint64_t active, uint64_t g) {
  if (g + 4 <= active) return *reinterpret_cast<const uint32_t*>(bva + g);
  uint32_t w = 0;
  for (int j = 0; j < 4; ++j)
    if (g + j < active) w |= uint32_t(uint8_t(bva[g + j])) << (8 * j);
  return w;
}

constexpr int kMmaThreads = 256;                // 8 warps
constexpr int kMmaWarps = kMmaThreads / 32;
constexpr int kMmaTiles = 4;                    // 16-row tiles per warp and iteration
constexpr int kMmaRows = 16 * kMmaTiles;        // output rows per warp and iteration

// Writes a warp's output rows from its s32 limb sums: acc[q][nt] is the
// accumulator of row tile q, column tile nt; with add_prev the previous
// value is added.  The quad of lanes that shares a row holds its 8
// coefficients (t and t + 4 per lane); they meet in shared memory and leave
// as one 16-byte store per row.
__device__ __forceinline__ void mma_store_rows(uint16_t (*out_s)[8], const int32_t (&acc)[kMmaTiles][2][4], uint64_t row0,
                                               uint64_t rows, Fe* __restrict__ dst, bool add_prev) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int q = 0; q < kMmaTiles; ++q) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // row g, then g + 8
      const int r = q * 16 + g + 8 * h;
      out_s[r][t] = uint16_t(mod_i64(int64_t(acc[q][0][2 * h]) + 256 * int64_t(acc[q][0][2 * h + 1])));
      out_s[r][t + 4] = uint16_t(mod_i64(int64_t(acc[q][1][2 * h]) + 256 * int64_t(acc[q][1][2 * h + 1])));
    }
  }
  __syncwarp();
  for (int r = lane; r < kMmaRows; r += 32) {
    const uint64_t row = row0 + r;
    if (row >= rows) continue;
    Fr v = unpack_fe(*reinterpret_cast<const uint4*>(out_s[r]));
    if (add_prev) v = add(load(dst + row), v);
    store(dst + row, v);
  }
  __syncwarp();
}

// Packed EO witness for stride 16: witness[row] = sum_{lane < 16}
// v(16 row + lane) * inv_powers[lane].  A = the weights (row-major: a row's
// 16 entries are contiguous), B = the limbs of the 16 powers; one k16 product
// per 16 rows and column tile.  |limb sum| < 16 * 128 * 255, so each
// coefficient sum is below 2^27.
__global__ void __launch_bounds__(kMmaThreads) k_eo_witness_mma(const int8_t* __restrict__ bva, uint64_t active,
                                                                uint64_t rows, const Fe* __restrict__ inv_powers,
                                                                Fe* __restrict__ witness) {
  __shared__ __align__(16) uint16_t out_s[kMmaWarps][kMmaRows][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  uint32_t bf[2];
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    uint32_t w = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) w |= fe_limb(inv_powers + 4 * t + e, nt * 8 + g) << (8 * e);
    bf[nt] = w;
  }
  const uint64_t wid = uint64_t(blockIdx.x) * kMmaWarps + warp, nw = uint64_t(gridDim.x) * kMmaWarps;
  for (uint64_t row0 = wid * kMmaRows; row0 < rows; row0 += nw * kMmaRows) {
    uint32_t a[kMmaTiles][2];
#pragma unroll
    for (int q = 0; q < kMmaTiles; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint64_t row = row0 + q * 16 + g + 8 * h;
        a[q][h] = row < rows ? weight_word(bva, active, row * 16 + 4 * t) : 0u;
      }
    int32_t acc[kMmaTiles][2][4];
#pragma unroll
    for (int q = 0; q < kMmaTiles; ++q)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[q][nt][c] = 0;
        mma_s8u8_k16(acc[q][nt], a[q][0], a[q][1], bf[nt]);
      }
    mma_store_rows(out_s[warp], acc, row0, rows, witness, false);
  }
}

// Block fold: values[i] = sum_b sum_{j < 8} v(b * block_len + 8 i + j) *
// T[b * 8 + j] (+ values[i] when `accumulate`).  K runs over (block, lane)
// pairs, 64 per group of 8 blocks: two k32 products per column tile, each A
// register one aligned 32-bit word of 4 lanes of one block.  A group's limb
// sums are below 64 * 128 * 255 < 2^21, so s32 accumulators hold 2^9
// groups; the coefficient combination is formed in 64 bits.
__global__ void __launch_bounds__(kMmaThreads) k_block_fold_mma(const int8_t* __restrict__ bva, uint64_t active,
                                                                uint64_t block_len, int blocks, uint64_t m,
                                                                const Fe* __restrict__ T, Fe* __restrict__ values,
                                                                int accumulate) {
  __shared__ __align__(16) uint16_t out_s[kMmaWarps][kMmaRows][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int groups = (blocks + 7) / 8;
  const uint64_t wid = uint64_t(blockIdx.x) * kMmaWarps + warp, nw = uint64_t(gridDim.x) * kMmaWarps;
  for (uint64_t row0 = wid * kMmaRows; row0 < m; row0 += nw * kMmaRows) {
    int32_t acc[kMmaTiles][2][4];
#pragma unroll
    for (int q = 0; q < kMmaTiles; ++q)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[q][nt][c] = 0;
    for (int gr = 0; gr < groups; ++gr) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {  // blocks 8 gr + 4 s .. + 3
        // Register half r of the A / B fragments covers block
        // 8 gr + 4 s + 2 r + (t >> 1), lanes 4 (t & 1) .. + 3.
        int bk[2];
        uint32_t bf[2][2];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          bk[r] = 8 * gr + 4 * s + 2 * r + (t >> 1);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            uint32_t w = 0;
            if (bk[r] < blocks)
#pragma unroll
              for (int e = 0; e < 4; ++e) w |= fe_limb(T + bk[r] * 8 + 4 * (t & 1) + e, nt * 8 + g) << (8 * e);
            bf[nt][r] = w;
          }
        }
#pragma unroll
        for (int q = 0; q < kMmaTiles; ++q) {
          uint32_t a[4];
#pragma unroll
          for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const uint64_t i = row0 + q * 16 + g + 8 * h;
              a[2 * r + h] = (bk[r] < blocks && i < m)
                                 ? weight_word(bva, active, uint64_t(bk[r]) * block_len + 8 * i + 4 * (t & 1))
                                 : 0u;
            }
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) mma_s8u8_k32(acc[q][nt], a, bf[nt][0], bf[nt][1]);
        }
      }
    }
    mma_store_rows(out_s[warp], acc, row0, m, values, accumulate != 0);
  }
}

// Batch-opening lane sums of up to 8 blocks against the equality weights
// (project_lanes_from_fn, packed_batch.rs:25-41):
//   raw[b][j * 8 + k] += sum_i v(b, 8 i + j) * weights[i].c[k].
// The contraction runs over the element index i, which is the outer index
// of both the weights (8 lanes j per element) and the table (16 limbs per
// element), so each fragment register is gathered: four 32-bit loads (the
// word holding byte j, or limb l, of four consecutive elements) and three
// byte permutes.  Rows of the A tile are (block pair member, lane j): row g
// is lane g of the pair's first block, row g + 8 lane g of the second.  Per
// k32 step the limb sums are below 32 * 128 * 255 < 2^20; s32 accumulators
// run 256 steps before they move into 64-bit totals.
constexpr int kEqMmaSteps = 256;  // k32 steps between flushes into 64-bit totals
__device__ __forceinline__ uint32_t gather_bytes(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, int b) {
  const uint32_t sel = uint32_t(b) | (uint32_t(4 + b) << 4);
  return __byte_perm(__byte_perm(x0, x1, sel), __byte_perm(x2, x3, sel), 0x5410);
}
__global__ void __launch_bounds__(kMmaThreads) k_eq_project_mma(const int8_t* __restrict__ bva, uint64_t active,
                                                                uint64_t block_len, uint64_t first_block, int nb, uint64_t m,
                                                                const Fe* __restrict__ weights,
                                                                unsigned long long* __restrict__ raw) {
  __shared__ long long tot_s[8][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  for (int i = threadIdx.x; i < 8 * 64; i += kMmaThreads) tot_s[i >> 6][i & 63] = 0;
  __syncthreads();
  const int pairs = (nb + 1) / 2;
  int32_t acc[4][2][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[p][nt][c] = 0;
  const uint64_t steps = (m + 31) / 32;
  const uint64_t wid = uint64_t(blockIdx.x) * kMmaWarps + warp, nw = uint64_t(gridDim.x) * kMmaWarps;
  // Moves the s32 sums into the CTA's 64-bit totals: lane (g, t) holds, for
  // block 2p + h, lane j = g, coefficient nt * 4 + t.
  auto flush = [&]() {
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const int64_t v = int64_t(acc[p][nt][2 * h]) + 256 * int64_t(acc[p][nt][2 * h + 1]);
          acc[p][nt][2 * h] = acc[p][nt][2 * h + 1] = 0;
          if (2 * p + h < nb)
            atomicAdd(reinterpret_cast<unsigned long long*>(&tot_s[2 * p + h][g * 8 + nt * 4 + t]),
                      (unsigned long long)v);
        }
  };
  int since = 0;
  for (uint64_t st = wid; st < steps; st += nw) {
    const uint64_t i0 = st * 32;
    // B: limb nt * 8 + g of elements i0 + 16 r + 4 t + e (word 2 nt + g / 4).
    uint32_t bf[2][2];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        uint32_t x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const uint64_t i = i0 + 16 * r + 4 * t + e;
          x[e] = i < m ? reinterpret_cast<const uint32_t*>(weights + i)[2 * nt + (g >> 2)] : 0u;
        }
        bf[nt][r] = gather_bytes(x[0], x[1], x[2], x[3], g & 3);
      }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      if (p >= pairs) break;
      uint32_t a[4];
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int h = 0; h < 2; ++h) {  // A register 2 r + h: row half h (block 2p + h), K half r
          const int b = 2 * p + h;
          uint32_t x[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const uint64_t i = i0 + 16 * r + 4 * t + e;
            x[e] = (b < nb && i < m) ? weight_word(bva, active, (first_block + b) * block_len + 8 * i + 4 * (g >> 2)) : 0u;
          }
          a[2 * r + h] = gather_bytes(x[0], x[1], x[2], x[3], g & 3);
        }
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) mma_s8u8_k32(acc[p][nt], a, bf[nt][0], bf[nt][1]);
    }
    if (++since == kEqMmaSteps) {
      flush();
      since = 0;
    }
  }
  flush();
  __syncthreads();
  for (int i = threadIdx.x; i < nb * 64; i += kMmaThreads)
    atomicAdd(raw + i, (unsigned long long)tot_s[i >> 6][i & 63]);  // two's complement sum
}

}  // namespace QFD_NS
