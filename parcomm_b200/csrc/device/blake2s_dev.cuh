// BLAKE2s-256 compression on the device (RFC 7693), one message per thread.
// Rotations by 12 and 7 are single funnel shifts, those by 16 and 8 byte
// permutes.  (Rotations as the two halves of a 32 x 32 -> 64-bit product,
// moved to the FMA pipe, measured 35 % slower in the leaf pass.)
#pragma once
#include <cstdint>

namespace qfd {

static __constant__ uint32_t kIv[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};

__device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }
// Rotations by whole bytes as byte permutes (funnel shifts issue at half rate).
__device__ __forceinline__ uint32_t rotr16(uint32_t x) { return __byte_perm(x, x, 0x1032); }
__device__ __forceinline__ uint32_t rotr8(uint32_t x) { return __byte_perm(x, x, 0x0321); }
// a + b as a 32-bit multiply-add by `one` (a runtime 1 from the kernel's
// arguments): it issues to the FMA pipe, leaving the ALU pipe, which the
// XORs and rotations keep busy, to them.
__device__ __forceinline__ uint32_t add_fma(uint32_t a, uint32_t b, uint32_t one) {
  uint32_t d;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(b), "r"(one), "r"(a));
  return d;
}

#define QFD_G(a, b, c, d, x, y)                         \
  v[a] = add_fma(add_fma(v[a], v[b], one), (x), one);   \
  v[d] = rotr16(v[d] ^ v[a]);                           \
  v[c] = add_fma(v[c], v[d], one);                      \
  v[b] = rotr(v[b] ^ v[c], 12);                         \
  v[a] = add_fma(add_fma(v[a], v[b], one), (y), one);   \
  v[d] = rotr8(v[d] ^ v[a]);                            \
  v[c] = add_fma(v[c], v[d], one);                      \
  v[b] = rotr(v[b] ^ v[c], 7);

#define QFD_ROUND(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  QFD_G(0, 4, 8, 12, m[s0], m[s1]);                                                     \
  QFD_G(1, 5, 9, 13, m[s2], m[s3]);                                                     \
  QFD_G(2, 6, 10, 14, m[s4], m[s5]);                                                    \
  QFD_G(3, 7, 11, 15, m[s6], m[s7]);                                                    \
  QFD_G(0, 5, 10, 15, m[s8], m[s9]);                                                    \
  QFD_G(1, 6, 11, 12, m[s10], m[s11]);                                                  \
  QFD_G(2, 7, 8, 13, m[s12], m[s13]);                                                   \
  QFD_G(3, 4, 9, 14, m[s14], m[s15]);

// h <- compress(h, m, t, last); `one` must be 1.  The sigma schedule is
// unrolled so every message index is a compile-time constant.
__device__ __forceinline__ void compress(uint32_t h[8], const uint32_t m[16], uint32_t t, bool last, uint32_t one) {
  uint32_t v[16];
#pragma unroll
  for (int i = 0; i < 8; ++i) { v[i] = h[i]; v[i + 8] = kIv[i]; }
  v[12] ^= t;
  if (last) v[14] = ~v[14];
  QFD_ROUND(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15)
  QFD_ROUND(14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3)
  QFD_ROUND(11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4)
  QFD_ROUND(7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8)
  QFD_ROUND(9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13)
  QFD_ROUND(2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9)
  QFD_ROUND(12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11)
  QFD_ROUND(13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10)
  QFD_ROUND(6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5)
  QFD_ROUND(10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0)
#pragma unroll
  for (int i = 0; i < 8; ++i) h[i] ^= v[i] ^ v[i + 8];
}
#undef QFD_G
#undef QFD_ROUND

}  // namespace qfd
