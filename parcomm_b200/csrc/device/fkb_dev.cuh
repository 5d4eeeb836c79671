// Device arithmetic for KoalaBear (p = 2^31 - 2^24 + 1) and its quartic
// extension KoalaBear[X]/(X^4 - 3).
//
// Storage: 4 canonical u32 coefficients = 16 bytes, which is also the
// canonical little-endian wire encoding (koalabear.rs write_canonical_bytes),
// moved as one uint4.  Products reduce with a Barrett step on 64-bit values;
// results are canonical, so they match the host field bit for bit.
#pragma once
#include <cstdint>

#ifndef QFD_HD
#define QFD_HD __host__ __device__ __forceinline__
#endif

namespace qfdkb {

constexpr uint32_t P = 2130706433u;
constexpr int kC = 4;                                   // coefficients per element
constexpr uint64_t kBarrett = 8657571868ull;            // floor(2^64 / p)
using Wt = int16_t;                                     // one BVA entry

struct __align__(16) Fe {
  uint32_t c[4];
};

struct Fr {
  uint32_t c[4];
};

QFD_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return uint64_t((unsigned __int128)a * b >> 64);
#endif
}
// Any u64 to canonical: q = floor(v * floor(2^64/p) / 2^64) undershoots
// floor(v / p) by at most 2, so at most two subtractions remain.
QFD_HD uint32_t red64(uint64_t v) {
  uint64_t r = v - mulhi64(v, kBarrett) * P;
  if (r >= P) r -= P;
  if (r >= P) r -= P;
  return uint32_t(r);
}
QFD_HD uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }
QFD_HD uint32_t red32(uint32_t v) { return v >= P ? v - P : v; }  // v < 2p
// A signed v with |v| < 2^62: adding kBias (the multiple of p just above
// 2^62) gives the same residue as an unsigned value below 2^64.
constexpr uint64_t kBias = ((uint64_t(1) << 62) / P + 1) * P;
QFD_HD uint32_t red_signed(int64_t v) { return red64(uint64_t(v) + kBias); }
// Canonical a, b < p < 2^31.  The sum is below 2^32, and s - p wraps above
// s exactly when s < p, so the unsigned minimum picks the reduced value; for
// the difference, a - b wraps above a - b + p exactly when a < b.
QFD_HD uint32_t addp(uint32_t a, uint32_t b) {
  const uint32_t s = a + b;
  return umin32(s, s - P);
}
QFD_HD uint32_t subp(uint32_t a, uint32_t b) {
  const uint32_t d = a - b;
  return umin32(d, d + P);
}

QFD_HD Fr unpack_fe(uint4 u) { Fr r; r.c[0] = u.x; r.c[1] = u.y; r.c[2] = u.z; r.c[3] = u.w; return r; }
QFD_HD uint4 pack_fe(const Fr& r) { return make_uint4(r.c[0], r.c[1], r.c[2], r.c[3]); }
QFD_HD Fr load(const Fe* p) { return unpack_fe(*reinterpret_cast<const uint4*>(p)); }
QFD_HD void store(Fe* p, const Fr& r) { *reinterpret_cast<uint4*>(p) = pack_fe(r); }
QFD_HD Fr zero() { Fr r; for (int i = 0; i < 4; ++i) r.c[i] = 0; return r; }
QFD_HD Fr add(const Fr& a, const Fr& b) { Fr r; for (int i = 0; i < 4; ++i) r.c[i] = addp(a.c[i], b.c[i]); return r; }
QFD_HD Fr sub(const Fr& a, const Fr& b) { Fr r; for (int i = 0; i < 4; ++i) r.c[i] = subp(a.c[i], b.c[i]); return r; }
QFD_HD Fr mul(const Fr& a, const Fr& b) {
  // X^4 = 3: the wrap-around products take 3 * b_j mod p, so output
  // coefficient k is one sum of four products < 2^62, i.e. below 2^64.
  uint32_t b3[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) b3[j] = addp(addp(b.c[j], b.c[j]), b.c[j]);
  uint64_t r[4] = {0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (i + j < 4) r[i + j] += uint64_t(a.c[i]) * b.c[j];
      else r[i + j - 4] += uint64_t(a.c[i]) * b3[j];
    }
  Fr out;
#pragma unroll
  for (int k = 0; k < 4; ++k) out.c[k] = red64(r[k]);
  return out;
}
// Sums of products: one product already fills a 64-bit raw coefficient, so
// each product is reduced and added (the F65521 header keeps them lazy).
struct Acc {
  Fr v;
};
QFD_HD Acc acc_zero() { Acc r; r.v = zero(); return r; }
QFD_HD void mul_acc(Acc& r, const Fr& a, const Fr& b) { r.v = add(r.v, mul(a, b)); }
QFD_HD Fr acc_reduce(const Acc& r) { return r.v; }
QFD_HD Fr mul_base(const Fr& a, uint32_t s) {
  Fr r;
  for (int i = 0; i < 4; ++i) r.c[i] = red64(uint64_t(a.c[i]) * s);
  return r;
}
// small signed integer -> canonical KoalaBear (field.rs:25-29)
QFD_HD uint32_t small(int v) { return v < 0 ? uint32_t(int64_t(v) + P) : uint32_t(v); }
// Σ of kC products of canonical values (< 2^64) to canonical.
QFD_HD uint32_t red_sum(uint64_t v) { return red64(v); }

// Planar transform tiles: every butterfly output is reduced right away (2p
// fits 32 bits, 2^l p does not), so the lazy bound is unused.
QFD_HD uint32_t tile_bound(int) { return P; }
QFD_HD void bfly_wht(uint32_t& lo, uint32_t& hi, uint32_t) {
  const uint32_t a = lo, b = hi;
  lo = addp(a, b);
  hi = subp(a, b);
}
QFD_HD void bfly_mobius(uint32_t lo, uint32_t& hi, uint32_t) { hi = subp(hi, lo); }
QFD_HD uint32_t tile_final(uint32_t v) { return v; }
// Four signed 16-bit payloads (8 bytes) to the packed element.
QFD_HD Fr weights_to_fr(uint2 raw) {
  Fr r;
  r.c[0] = small(int(int16_t(raw.x & 0xffffu)));
  r.c[1] = small(int(int16_t(raw.x >> 16)));
  r.c[2] = small(int(int16_t(raw.y & 0xffffu)));
  r.c[3] = small(int(int16_t(raw.y >> 16)));
  return r;
}

}  // namespace qfdkb
