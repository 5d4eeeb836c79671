// LogUp range audit on the device: one pass over the BVA values that
// accumulates sum_i 1 / (alpha - v_i) as a fraction and counts each value's
// multiplicity over the entry type's table (int8: 256 values, int16: 65536).
//
// The fraction sum is formed per value, without the multiplicities: for each
// group of G values (8 int8 entries, 4 int16 entries) the polynomial
// P(x) = prod (x - v_j) is built with exact integer coefficients (|c_k| below
// 2^57 for eight int8 values, 2^61 for four int16 values), so that
// sum_j 1 / (alpha - v_j) = P'(alpha) / P(alpha).  P(alpha) and P'(alpha) take
// G base-by-extension products per coefficient lane from alpha^1..alpha^G
// (kernel parameters: constant-bank operands), and a running fraction n / d
// absorbs the group with three extension products: (n P + P' d) / (d P).
// Each thread keeps two running fractions (even and odd groups) so that two
// chains of extension products overlap.
//
// Multiplicities go to shared memory.  For int8, each warp keeps its own 256
// 32-bit counters.  The 65536 int16 counters are 16-bit halves of 32768
// words (128 KB); a CTA of 384 threads adds at most 64,519 values between
// flushes to the global 64-bit histogram, so a half never carries into its
// neighbour.
#pragma once
#include <cstdint>

#include "../device/field_dev.cuh"
#include "open.cuh"

namespace QFD_NS {

// 384 threads: the two product chains fit in registers (no spills).
constexpr int kAuditThreads = 384;
constexpr int kAuditPerChunk = 16 / int(sizeof(Wt));  // values per 16-byte load
constexpr int kAuditBins = sizeof(Wt) == 1 ? 256 : 65536;
constexpr int kAuditMin = sizeof(Wt) == 1 ? -128 : -32768;
constexpr int kAuditWarps = kAuditThreads / 32;
// int16: rounds of one chunk per thread between flushes of the 16-bit halves.
constexpr int kAuditEpochRounds = 65535 / (kAuditThreads * kAuditPerChunk);
constexpr size_t kAuditSmemWords = sizeof(Wt) == 1 ? size_t(kAuditWarps) * 256 : 32768;
constexpr size_t kAuditSmem = kAuditSmemWords * 4;
static_assert(sizeof(Wt) == 1 || size_t(kAuditEpochRounds) * kAuditThreads * kAuditPerChunk + kAuditPerChunk < 65536,
              "an epoch must stay below 2^16 values per CTA");
static_assert(kAuditSmemWords >= size_t(kAuditWarps) * 4 * kC, "fraction reduction reuses the counters");

constexpr int kAuditGroup = sizeof(Wt) == 1 ? 8 : 4;  // values per polynomial

// alpha^1 .. alpha^G as canonical 32-bit coefficient lanes.
struct AlphaPowers {
  uint32_t c[kAuditGroup][kC];
};

struct Frac {
  Fr n, d;
};

__device__ __forceinline__ Frac frac_add(const Frac& a, const Frac& b) {
  Acc t = acc_zero();
  mul_acc(t, a.n, b.d);
  mul_acc(t, b.n, a.d);
  return {acc_reduce(t), mul(a.d, b.d)};
}

// Coefficients q[0..4] of the monic quartic prod_{j<4} (x - v_j).
__device__ __forceinline__ void quartic(const int* v, long long* q) {
  const long long a1 = v[0] + v[1], a2 = (long long)v[0] * v[1], b1 = v[2] + v[3], b2 = (long long)v[2] * v[3];
  q[4] = 1;
  q[3] = -(a1 + b1);
  q[2] = a2 + b2 + a1 * b1;
  q[1] = -(a1 * b2 + a2 * b1);
  q[0] = a2 * b2;
}

// n / d += sum_j 1 / (alpha - v_j) over kAuditGroup values.
__device__ __forceinline__ void audit_group(Frac& f, const AlphaPowers& ap, const int* v) {
  constexpr int G = kAuditGroup;
  long long c[G + 1];  // P(x) = sum_k c[k] x^k, c[G] = 1
  if constexpr (G == 4) {
    quartic(v, c);
  } else {
    long long x[5], y[5];
    quartic(v, x);
    quartic(v + 4, y);
#pragma unroll
    for (int k = 0; k <= 8; ++k) c[k] = 0;
#pragma unroll
    for (int i = 0; i <= 4; ++i)
#pragma unroll
      for (int j = 0; j <= 4; ++j) c[i + j] += x[i] * y[j];
  }
  // P(alpha) = alpha^G + sum_{k<G} c_k alpha^k and P'(alpha) = G alpha^(G-1) +
  // sum_{1<=k<G} k c_k alpha^(k-1): per lane, products below 2^62 (KoalaBear:
  // at most three of them and two canonical terms in one 64-bit sum; F65521:
  // products below 2^35).
  uint32_t m[G];
#pragma unroll
  for (int k = 0; k < G; ++k) m[k] = red_signed(c[k]);
  Fr P, D;
#pragma unroll
  for (int j = 0; j < kC; ++j) {
    uint64_t s = ap.c[G - 1][j], t;
    if constexpr (sizeof(Wt) == 1) {
      t = uint64_t(G) * ap.c[G - 2][j];
#pragma unroll
      for (int k = 1; k < G; ++k) s += uint64_t(m[k]) * ap.c[k - 1][j];
#pragma unroll
      for (int k = 2; k < G; ++k) t += uint64_t(k * m[k]) * ap.c[k - 2][j];
      if (j == 0) { s += m[0]; t += m[1]; }
      P.c[j] = red_sum(s);
      D.c[j] = red_sum(t);
    } else {
      // G = 4: P = a^4 + m3 a^3 + m2 a^2 + m1 a + m0, P' = 4 a^3 + 3 m3 a^2 + 2 m2 a + m1.
      s += uint64_t(m[3]) * ap.c[2][j] + uint64_t(m[2]) * ap.c[1][j] + uint64_t(m[1]) * ap.c[0][j];
      t = 4ull * ap.c[2][j] + uint64_t(red_signed(3 * c[3])) * ap.c[1][j] + uint64_t(red_signed(2 * c[2])) * ap.c[0][j];
      if (j == 0) { s += m[0]; t += m[1]; }
      P.c[j] = red_sum(s);
      D.c[j] = red_sum(t);
    }
  }
  Acc t = acc_zero();
  mul_acc(t, f.n, P);
  mul_acc(t, D, f.d);
  f.n = acc_reduce(t);
  f.d = mul(f.d, P);
}

// n / d += 1 / (alpha - v).
__device__ __forceinline__ void audit_one(Frac& f, const Fr& alpha, int v) {
  Fr q = alpha;
  q.c[0] = subp(q.c[0], small(v));
  f.n = add(mul(f.n, q), f.d);
  f.d = mul(f.d, q);
}

__device__ __forceinline__ void audit_count(uint32_t* wb, int v) {
  const uint32_t idx = uint32_t(v - kAuditMin);
  if constexpr (sizeof(Wt) == 1) atomicAdd(wb + idx, 1u);
  else atomicAdd(wb + (idx >> 1), (idx & 1u) ? 0x10000u : 1u);
}

// Adds the shared int16 counters to `hist` and clears them (whole CTA).
__device__ __forceinline__ void audit_flush16(uint32_t* bins, unsigned long long* hist) {
  __syncthreads();
  for (uint32_t w = threadIdx.x; w < 32768; w += blockDim.x) {
    const uint32_t x = bins[w];
    if (x) {
      bins[w] = 0;
      if (x & 0xffffu) atomicAdd(hist + 2 * w, (unsigned long long)(x & 0xffffu));
      if (x >> 16) atomicAdd(hist + 2 * w + 1, (unsigned long long)(x >> 16));
    }
  }
  __syncthreads();
}

// One launch over n values (16-byte aligned).  Adds the multiplicities to
// hist[kAuditBins] (bin k counts the value k + kAuditMin) and writes this
// CTA's fraction to partials[2 * blockIdx.x] (numerator, denominator).
__global__ void __launch_bounds__(kAuditThreads, 1)
k_range_audit(const Wt* __restrict__ vals, uint64_t n, AlphaPowers ap, unsigned long long* __restrict__ hist,
              Fe* __restrict__ partials) {
  extern __shared__ uint32_t bins[];
  for (uint32_t i = threadIdx.x; i < kAuditSmemWords; i += blockDim.x) bins[i] = 0;
  __syncthreads();
  Frac f[2] = {{zero(), zero()}, {zero(), zero()}};
  f[0].d.c[0] = f[1].d.c[0] = 1;
  uint32_t* wb = sizeof(Wt) == 1 ? bins + (threadIdx.x >> 5) * 256 : bins;
  const uint64_t chunks = n / kAuditPerChunk;
  const uint64_t per_round = uint64_t(gridDim.x) * kAuditThreads;
  const uint64_t rounds = (chunks + per_round - 1) / per_round;
  const uint4* src = reinterpret_cast<const uint4*>(vals);
  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t c = r * per_round + uint64_t(blockIdx.x) * kAuditThreads + threadIdx.x;
    if (c < chunks) {
      const uint4 u = __ldg(src + c);
      const uint32_t w[4] = {u.x, u.y, u.z, u.w};
      int v[kAuditPerChunk];
#pragma unroll
      for (int i = 0; i < kAuditPerChunk; ++i) {
        if constexpr (sizeof(Wt) == 1) v[i] = int(int8_t(w[i >> 2] >> (8 * (i & 3))));
        else v[i] = int(int16_t(w[i >> 1] >> (16 * (i & 1))));
      }
      static_assert(kAuditPerChunk == 2 * kAuditGroup, "two groups per 16-byte chunk");
      audit_group(f[0], ap, v);
      audit_group(f[1], ap, v + kAuditGroup);
#pragma unroll
      for (int i = 0; i < kAuditPerChunk; ++i) audit_count(wb, v[i]);
    }
    if constexpr (sizeof(Wt) == 2)
      if ((r + 1) % kAuditEpochRounds == 0) audit_flush16(bins, hist);  // uniform over the CTA
  }
  // The last n % kAuditPerChunk values, one at a time.
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (uint64_t i = chunks * kAuditPerChunk; i < n; ++i) {
      const int v = int(vals[i]);
      Fr alpha;
#pragma unroll
      for (int j = 0; j < kC; ++j) alpha.c[j] = ap.c[0][j];
      audit_one(f[0], alpha, v);
      audit_count(wb, v);
    }
  if constexpr (sizeof(Wt) == 2) {
    audit_flush16(bins, hist);
  } else {
    __syncthreads();
    if (threadIdx.x < 256) {
      unsigned long long s = 0;
      for (int w = 0; w < kAuditWarps; ++w) s += bins[w * 256 + threadIdx.x];
      if (s) atomicAdd(hist + threadIdx.x, s);
    }
    __syncthreads();
  }
  // Fraction sum over the CTA: the thread's two, lanes, then warps (through
  // the counters' memory).
  Frac t = frac_add(f[0], f[1]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Frac g{shfl_xor(t.n, o), shfl_xor(t.d, o)};
    t = frac_add(t, g);
  }
  Fr* red = reinterpret_cast<Fr*>(bins);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[2 * warp] = t.n; red[2 * warp + 1] = t.d; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kAuditWarps; ++w) t = frac_add(t, Frac{red[2 * w], red[2 * w + 1]});
    store(partials + 2 * blockIdx.x, t.n);
    store(partials + 2 * blockIdx.x + 1, t.d);
  }
}

}  // namespace QFD_NS
