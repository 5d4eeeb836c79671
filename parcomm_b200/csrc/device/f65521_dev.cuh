// Device arithmetic for F_65521 and F_65521[X]/(X^8 - 17).
//
// Storage: 8 canonical u16 coefficients = 16 bytes, moved as one uint4
// (one 128-bit load/store per element).  Arithmetic unpacks to 32-bit
// registers.  Reductions use 2^16 = 15 (mod p) twice, the same
// pseudo-Mersenne identity as Prime65521::reduce_u32 (qafold_short.rs:336-346);
// results are canonical, so they match the host field bit for bit.
#pragma once
#include <cstdint>

namespace qfd {

constexpr uint32_t P = 65521u;

struct __align__(16) Fe {
  uint16_t c[8];
};

// Register form: eight canonical coefficients in 32-bit lanes.
struct Fr {
  uint32_t c[8];
};

__device__ __forceinline__ uint32_t red32(uint32_t v) {
  uint32_t f = (v & 0xffffu) + 15u * (v >> 16);
  f = (f & 0xffffu) + 15u * (f >> 16);
  return f >= P ? f - P : f;
}
__device__ __forceinline__ uint32_t red64(uint64_t v) {  // v < 2^48
  uint64_t f = (v & 0xffffu) + 15ull * (v >> 16);
  uint32_t g = uint32_t((f & 0xffffu) + 15ull * (f >> 16));
  return red32(g);
}
__device__ __forceinline__ uint32_t addp(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P ? s - P : s; }
__device__ __forceinline__ uint32_t subp(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }

__device__ __forceinline__ Fr load(const Fe* p) {
  uint4 u = *reinterpret_cast<const uint4*>(p);
  Fr r;
  r.c[0] = u.x & 0xffffu; r.c[1] = u.x >> 16;
  r.c[2] = u.y & 0xffffu; r.c[3] = u.y >> 16;
  r.c[4] = u.z & 0xffffu; r.c[5] = u.z >> 16;
  r.c[6] = u.w & 0xffffu; r.c[7] = u.w >> 16;
  return r;
}
__device__ __forceinline__ void store(Fe* p, const Fr& r) {
  uint4 u;
  u.x = r.c[0] | (r.c[1] << 16);
  u.y = r.c[2] | (r.c[3] << 16);
  u.z = r.c[4] | (r.c[5] << 16);
  u.w = r.c[6] | (r.c[7] << 16);
  *reinterpret_cast<uint4*>(p) = u;
}
__device__ __forceinline__ Fr zero() { Fr r; for (int i = 0; i < 8; ++i) r.c[i] = 0; return r; }
__device__ __forceinline__ Fr add(const Fr& a, const Fr& b) { Fr r; for (int i = 0; i < 8; ++i) r.c[i] = addp(a.c[i], b.c[i]); return r; }
__device__ __forceinline__ Fr sub(const Fr& a, const Fr& b) { Fr r; for (int i = 0; i < 8; ++i) r.c[i] = subp(a.c[i], b.c[i]); return r; }
__device__ __forceinline__ Fr mul(const Fr& a, const Fr& b) {
  // Low and high product halves accumulate separately; the high half is
  // folded with X^8 = 17.  Each half-sum is < 8 * 65520^2 < 2^35.
  uint64_t lo[8], hi[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) { lo[k] = 0; hi[k] = 0; }
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t p = a.c[i] * b.c[j];
      if (i + j < 8) lo[i + j] += p; else hi[i + j - 8] += p;
    }
  Fr r;
#pragma unroll
  for (int k = 0; k < 8; ++k) r.c[k] = red64(lo[k] + 17ull * hi[k]);
  return r;
}
__device__ __forceinline__ Fr mul_base(const Fr& a, uint32_t s) {
  Fr r;
  for (int i = 0; i < 8; ++i) r.c[i] = red32(a.c[i] * s);
  return r;
}
// small signed integer -> canonical F_65521 (field.rs:24-26)
__device__ __forceinline__ uint32_t small(int v) { return v < 0 ? uint32_t(v + int(P)) : uint32_t(v); }

}  // namespace qfd
