// LogUp range audit on the device: one pass over the BVA values that
// accumulates sum_i 1 / (alpha - v_i) as a fraction and counts each value's
// multiplicity over the entry type's table (int8: 256 values, int16: 65536).
//
// The fraction sum is formed per value, without the multiplicities: for each
// group of four values the polynomial P(x) = prod (x - v_j) is built with
// exact integer coefficients (elementary symmetric sums, |e_4| < 2^61 for
// int16), so that sum_j 1 / (alpha - v_j) = P'(alpha) / P(alpha).  P(alpha)
// and P'(alpha) take three base-by-extension products per coefficient lane
// from alpha^1..alpha^4, and the running fraction n / d absorbs the group
// with three extension products: (n P + P' d) / (d P).
//
// Multiplicities go to shared memory.  For int8, each warp keeps its own 256
// 32-bit counters.  The 65536 int16 counters are 16-bit halves of 32768
// words (128 KB); a CTA adds at most 61,447 values between flushes to the
// global 64-bit histogram, so a half never carries into its neighbour.
#pragma once
#include <cstdint>

#include "../device/field_dev.cuh"
#include "open.cuh"

namespace QFD_NS {

constexpr int kAuditThreads = 512;
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

struct AlphaPowers {
  Fe p[4];  // alpha^1 .. alpha^4
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

// n / d += sum_j 1 / (alpha - v_j) over four values.
__device__ __forceinline__ void audit_group(Frac& f, const Fr (&a)[4], int v0, int v1, int v2, int v3) {
  const long long a1 = v0 + v1, a2 = (long long)v0 * v1, b1 = v2 + v3, b2 = (long long)v2 * v3;
  const long long e1 = a1 + b1, e2 = a2 + b2 + a1 * b1, e3 = a1 * b2 + a2 * b1, e4 = a2 * b2;
  // P(x) = x^4 - e1 x^3 + e2 x^2 - e3 x + e4, P'(x) = 4 x^3 - 3 e1 x^2 + 2 e2 x - e3.
  const uint32_t k3 = red_signed(-e1), k2 = red_signed(e2), k1 = red_signed(-e3), k0 = red_signed(e4);
  const uint32_t d2 = red_signed(-3 * e1), d1 = red_signed(2 * e2);
  Fr P, D;
#pragma unroll
  for (int j = 0; j < kC; ++j) {
    uint64_t s = uint64_t(a[3].c[j]) + uint64_t(k3) * a[2].c[j] + uint64_t(k2) * a[1].c[j] + uint64_t(k1) * a[0].c[j];
    uint64_t t = 4ull * a[2].c[j] + uint64_t(d2) * a[1].c[j] + uint64_t(d1) * a[0].c[j];
    if (j == 0) { s += k0; t += k1; }
    P.c[j] = red_sum(s);
    D.c[j] = red_sum(t);
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
  Fr a[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) a[k] = load(&ap.p[k]);
  Frac f{zero(), zero()};
  f.d.c[0] = 1;
  uint32_t* wb = sizeof(Wt) == 1 ? bins + (threadIdx.x >> 5) * 256 : bins;
  const uint64_t chunks = n / kAuditPerChunk;
  const uint64_t per_round = uint64_t(gridDim.x) * kAuditThreads;
  const uint64_t rounds = (chunks + per_round - 1) / per_round;
  const uint4* src = reinterpret_cast<const uint4*>(vals);
  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t c = r * per_round + uint64_t(blockIdx.x) * kAuditThreads + threadIdx.x;
    if (c < chunks) {
      // Four values per group: one word of int8 entries, two of int16.  The
      // groups run one after the other (words rotate down) to keep few live.
      uint4 u = __ldg(src + c);
#pragma unroll 1
      for (int g = 0; g < kAuditPerChunk / 4; ++g) {
        int v[4];
        if constexpr (sizeof(Wt) == 1) {
#pragma unroll
          for (int i = 0; i < 4; ++i) v[i] = int(int8_t(u.x >> (8 * i)));
          u = make_uint4(u.y, u.z, u.w, 0);
        } else {
          v[0] = int(int16_t(u.x)); v[1] = int(int16_t(u.x >> 16));
          v[2] = int(int16_t(u.y)); v[3] = int(int16_t(u.y >> 16));
          u = make_uint4(u.z, u.w, 0, 0);
        }
        audit_group(f, a, v[0], v[1], v[2], v[3]);
#pragma unroll
        for (int i = 0; i < 4; ++i) audit_count(wb, v[i]);
      }
    }
    if constexpr (sizeof(Wt) == 2)
      if ((r + 1) % kAuditEpochRounds == 0) audit_flush16(bins, hist);  // uniform over the CTA
  }
  // The last n % kAuditPerChunk values, one at a time.
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (uint64_t i = chunks * kAuditPerChunk; i < n; ++i) {
      const int v = int(vals[i]);
      audit_one(f, a[0], v);
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
  // Fraction sum over the CTA: lanes, then warps (through the counters' memory).
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Frac g{shfl_xor(f.n, o), shfl_xor(f.d, o)};
    f = frac_add(f, g);
  }
  Fr* red = reinterpret_cast<Fr*>(bins);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[2 * warp] = f.n; red[2 * warp + 1] = f.d; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kAuditWarps; ++w) f = frac_add(f, Frac{red[2 * w], red[2 * w + 1]});
    store(partials + 2 * blockIdx.x, f.n);
    store(partials + 2 * blockIdx.x + 1, f.d);
  }
}

}  // namespace QFD_NS
