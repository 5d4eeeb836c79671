// Device arithmetic for F_65521 and F_65521[X]/(X^8 - 17).
//
// Storage: 8 canonical u16 coefficients = 16 bytes, moved as one uint4
// (one 128-bit load/store per element).  Arithmetic unpacks to 32-bit
// registers.  Reductions use 2^16 = 15 (mod p) twice, the same
// pseudo-Mersenne identity as Prime65521::reduce_u32 (qafold_short.rs:336-346);
// results are canonical, so they match the host field bit for bit.
#pragma once
#include <cstdint>

// Host-callable too, so the arithmetic can be checked against the host field on a CPU.
#define QFD_HD __host__ __device__ __forceinline__

namespace qfd {

constexpr uint32_t P = 65521u;
constexpr int kC = 8;   // coefficients per element
using Wt = int8_t;      // one BVA entry

struct __align__(16) Fe {
  uint16_t c[8];
};

// Register form: eight canonical coefficients in 32-bit lanes.
struct Fr {
  uint32_t c[8];
};

QFD_HD uint32_t red32(uint32_t v) {
  uint32_t f = (v & 0xffffu) + 15u * (v >> 16);
  f = (f & 0xffffu) + 15u * (f >> 16);
  return f >= P ? f - P : f;
}
QFD_HD uint32_t red64(uint64_t v) {  // v < 2^48
  uint64_t f = (v & 0xffffu) + 15ull * (v >> 16);
  uint32_t g = uint32_t((f & 0xffffu) + 15ull * (f >> 16));
  return red32(g);
}
QFD_HD uint32_t addp(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P ? s - P : s; }
QFD_HD uint32_t subp(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }

QFD_HD Fr load(const Fe* p) {
  uint4 u = *reinterpret_cast<const uint4*>(p);
  Fr r;
  r.c[0] = u.x & 0xffffu; r.c[1] = u.x >> 16;
  r.c[2] = u.y & 0xffffu; r.c[3] = u.y >> 16;
  r.c[4] = u.z & 0xffffu; r.c[5] = u.z >> 16;
  r.c[6] = u.w & 0xffffu; r.c[7] = u.w >> 16;
  return r;
}
QFD_HD void store(Fe* p, const Fr& r) {
  uint4 u;
  u.x = r.c[0] | (r.c[1] << 16);
  u.y = r.c[2] | (r.c[3] << 16);
  u.z = r.c[4] | (r.c[5] << 16);
  u.w = r.c[6] | (r.c[7] << 16);
  *reinterpret_cast<uint4*>(p) = u;
}
QFD_HD Fr zero() { Fr r; for (int i = 0; i < 8; ++i) r.c[i] = 0; return r; }
QFD_HD Fr add(const Fr& a, const Fr& b) { Fr r; for (int i = 0; i < 8; ++i) r.c[i] = addp(a.c[i], b.c[i]); return r; }
QFD_HD Fr sub(const Fr& a, const Fr& b) { Fr r; for (int i = 0; i < 8; ++i) r.c[i] = subp(a.c[i], b.c[i]); return r; }
// v < 2^40 to canonical: two 2^16 = 15 folds (< 2^28 + 2^16, then < 2p) and
// one conditional subtraction.
QFD_HD uint32_t red40(uint64_t v) {
  uint32_t f = uint32_t(v & 0xffffu) + 15u * uint32_t(v >> 16);
  f = (f & 0xffffu) + 15u * (f >> 16);
  return f >= P ? f - P : f;
}
// A signed v with |v| < 2^62: adding kBias (the multiple of p just above
// 2^62) gives an unsigned value below 2^64 with the same residue; two folds
// of 2^16 = 15 bring it below 2^40 for red40.
constexpr uint64_t kBias = ((uint64_t(1) << 62) / P + 1) * P;
QFD_HD uint32_t red_signed(int64_t v) {
  uint64_t u = uint64_t(v) + kBias;
  u = (u & 0xffffu) + 15u * (u >> 16);
  u = (u & 0xffffu) + 15u * (u >> 16);
  return red40(u);
}
QFD_HD Fr mul(const Fr& a, const Fr& b) {
  // A loop's fixed factor goes second, so that 17 * b is computed once.
  // X^8 = 17: the wrap-around products take 17 * b_j (< 2^21, unreduced), so
  // output coefficient k is one sum of eight products a_i * b'_j < 2^37,
  // accumulated with 64-bit multiply-adds (< 2^40) and reduced once.
  uint32_t b17[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) b17[j] = 17u * b.c[j];
  uint64_t r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (i + j < 8) r[i + j] += uint64_t(a.c[i]) * b.c[j];
      else r[i + j - 8] += uint64_t(a.c[i]) * b17[j];
    }
  Fr out;
#pragma unroll
  for (int k = 0; k < 8; ++k) out.c[k] = red40(r[k]);
  return out;
}
// Lazy sums of products: a product adds at most eight terms below 2^36.1 to
// each raw coefficient (below 2^39.1), so a 64-bit accumulator takes 2^24
// products before it could overflow; it is reduced once at the end (two
// folds of 2^16 = 15 bring any u64 below 2^40, then red40).
struct Acc {
  uint64_t c[8];
};
QFD_HD Acc acc_zero() { Acc r; for (int k = 0; k < 8; ++k) r.c[k] = 0; return r; }
QFD_HD void mul_acc(Acc& r, const Fr& a, const Fr& b) {
  uint32_t b17[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) b17[j] = 17u * b.c[j];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (i + j < 8) r.c[i + j] += uint64_t(a.c[i]) * b.c[j];
      else r.c[i + j - 8] += uint64_t(a.c[i]) * b17[j];
    }
}
QFD_HD Fr acc_reduce(const Acc& r) {
  Fr out;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    uint64_t v = (r.c[k] & 0xffffu) + 15u * (r.c[k] >> 16);
    v = (v & 0xffffu) + 15u * (v >> 16);
    out.c[k] = red40(v);
  }
  return out;
}
QFD_HD Fr mul_base(const Fr& a, uint32_t s) {
  Fr r;
  for (int i = 0; i < 8; ++i) r.c[i] = red32(a.c[i] * s);
  return r;
}
// Σ of kC products of canonical values (< 2^35) to canonical.
QFD_HD uint32_t red_sum(uint64_t v) { return red64(v); }
QFD_HD Fr unpack_fe(uint4 u) {
  Fr v;
  v.c[0] = u.x & 0xffffu; v.c[1] = u.x >> 16; v.c[2] = u.y & 0xffffu; v.c[3] = u.y >> 16;
  v.c[4] = u.z & 0xffffu; v.c[5] = u.z >> 16; v.c[6] = u.w & 0xffffu; v.c[7] = u.w >> 16;
  return v;
}
QFD_HD uint4 pack_fe(const Fr& r) {
  return make_uint4(r.c[0] | (r.c[1] << 16), r.c[2] | (r.c[3] << 16), r.c[4] | (r.c[5] << 16), r.c[6] | (r.c[7] << 16));
}

// Planar transform tiles use lazy reduction: a value entering level l of a
// pass is below tile_bound(l) = 2^l p, a difference is formed as a + 2^l p - b,
// so twelve levels stay below 2^28 and tile_final reduces once per pass.
QFD_HD uint32_t tile_bound(int lvl) { return P << lvl; }
QFD_HD void bfly_wht(uint32_t& lo, uint32_t& hi, uint32_t B) {
  const uint32_t a = lo, b = hi;
  lo = a + b;
  hi = a + B - b;
}
QFD_HD void bfly_mobius(uint32_t lo, uint32_t& hi, uint32_t B) { hi = hi + B - lo; }
// Values below 2^28 (at most twelve lazy levels) to canonical form.
QFD_HD uint32_t tile_final(uint32_t v) {
  const uint32_t f = (v & 0xffffu) + 15u * (v >> 16);  // < 2^16 + 15 * 2^12 < 2p
  return f >= P ? f - P : f;
}

// small signed integer -> canonical F_65521 (field.rs:24-26)
QFD_HD uint32_t small(int v) { return v < 0 ? uint32_t(v + int(P)) : uint32_t(v); }
// Eight signed 8-bit weights (8 bytes) to the packed element.
QFD_HD Fr weights_to_fr(uint2 raw) {
  Fr r;
#pragma unroll
  for (int k = 0; k < 8; ++k) r.c[k] = small(int(int8_t(((k < 4 ? raw.x : raw.y) >> (8 * (k & 3))) & 0xffu)));
  return r;
}

}  // namespace qfd
