// KoalaBear (p = 2^31 - 2^24 + 1) and its quartic extension KoalaBear[X]/(X^4 - 3),
// used directly as the QAFold message field for 16-bit payloads.
//
// Reference: koalabear/vendor/qafold/src/koalabear.rs: KoalaBear (NAME
// "KoalaBear/scalar/v1", MODULUS 2130706433), KoalaBearExt4 (coordinates
// [1, X, X^2, X^3] with X^4 = 3, Frobenius phases [1, 2113994754, 2130706432,
// 16711679], canonical 16-byte little-endian encoding of four u32, uniform
// sampling by clearing the top bit of each word and rejecting values >= p,
// NAME "FullKoalaBearExt4/X^4-3/scalar/v1"); packed_koalabear.rs (four lanes,
// magic "QAKOAPK1", lane root of unity 2113994754); protocol and transcript
// domains of qafold/koalabear/src (transcript.rs:15, protocol.rs:330).
// Arithmetic is exact, so any correct reduction order gives identical
// canonical results.
#pragma once
#include <cstdint>
#include <cstring>

#include "field65521.h"  // QF_HD

namespace qf {

static constexpr uint32_t PKB = 2130706433u;  // 2^31 - 2^24 + 1

QF_HD uint32_t kb_reduce64(uint64_t v) { return uint32_t(v % PKB); }
QF_HD uint32_t kb_add(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= PKB ? s - PKB : s; }
QF_HD uint32_t kb_sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + PKB - b; }
QF_HD uint32_t kb_mul(uint32_t a, uint32_t b) { return kb_reduce64(uint64_t(a) * b); }
QF_HD uint32_t kb_neg(uint32_t a) { return a == 0 ? 0 : PKB - a; }
inline uint32_t kb_pow(uint32_t a, uint64_t e) {
  uint32_t r = 1;
  while (e) { if (e & 1) r = kb_mul(r, a); a = kb_mul(a, a); e >>= 1; }
  return r;
}
inline uint32_t kb_inv(uint32_t a) { return kb_pow(a, PKB - 2); }

struct Kb4 {
  using Coeff = uint32_t;
  uint32_t c[4];
  // Packed-PCS transcript domain and single-block proof magic (packed_koalabear.rs:25, 478).
  static constexpr const char* kPackedDomain = "mikros/qafold-koalabear-ext4/packed-boolean-mle/v1";
  static constexpr const char* kPackedMagic = "QAKOAPK1";
  // Outer protocol transcript and opening-context domains (transcript.rs:15, protocol.rs:330).
  static constexpr const char* kPublicDomain = "parcomm-koalabear-i16/public/v1";
  static constexpr const char* kTerminalDomain = "parcomm/koalabear-i16/terminal/v2";
  static uint32_t base_mul(uint32_t a, uint32_t b) { return kb_mul(a, b); }
  static uint32_t base_inv(uint32_t a) { return kb_inv(a % PKB); }
  // The primitive 4th root of unity of the lane DFT (packed_koalabear.rs:515), inverted.
  static uint32_t root_of_unity_inverse() { return kb_inv(2113994754u); }

  static constexpr int kLanes = 4;  // base values packed per element
  static constexpr uint32_t kPrime = PKB;
  static constexpr const char* kName = "FullKoalaBearExt4/X^4-3/scalar/v1";
  static unsigned __int128 cardinality() {
    unsigned __int128 r = 1;
    for (int i = 0; i < 4; ++i) r *= PKB;
    return r;
  }

  QF_HD static Kb4 zero() { Kb4 r; for (int i = 0; i < 4; ++i) r.c[i] = 0; return r; }
  QF_HD static Kb4 one() { Kb4 r = zero(); r.c[0] = 1; return r; }
  QF_HD static Kb4 from_base(uint32_t v) { Kb4 r = zero(); r.c[0] = v; return r; }
  QF_HD bool is_zero() const { for (int i = 0; i < 4; ++i) if (c[i]) return false; return true; }
  QF_HD bool operator==(const Kb4& o) const { for (int i = 0; i < 4; ++i) if (c[i] != o.c[i]) return false; return true; }
  QF_HD bool operator!=(const Kb4& o) const { return !(*this == o); }
  QF_HD Kb4 operator+(const Kb4& o) const { Kb4 r; for (int i = 0; i < 4; ++i) r.c[i] = kb_add(c[i], o.c[i]); return r; }
  QF_HD Kb4 operator-(const Kb4& o) const { Kb4 r; for (int i = 0; i < 4; ++i) r.c[i] = kb_sub(c[i], o.c[i]); return r; }
  QF_HD Kb4 operator-() const { Kb4 r; for (int i = 0; i < 4; ++i) r.c[i] = kb_neg(c[i]); return r; }
  QF_HD Kb4& operator+=(const Kb4& o) { *this = *this + o; return *this; }
  QF_HD Kb4& operator-=(const Kb4& o) { *this = *this - o; return *this; }
  QF_HD Kb4 operator*(const Kb4& o) const {
    // Schoolbook with X^4 = 3: each product is reduced to < p first, so a
    // coefficient sums at most 4 values < p plus 3 times 3 more (< 2^35).
    uint64_t acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        const uint64_t p = kb_mul(c[i], o.c[j]);
        const int k = i + j;
        if (k < 4) acc[k] += p; else acc[k - 4] += 3u * p;
      }
    Kb4 r;
    for (int k = 0; k < 4; ++k) r.c[k] = kb_reduce64(acc[k]);
    return r;
  }
  QF_HD Kb4& operator*=(const Kb4& o) { *this = *this * o; return *this; }
  QF_HD Kb4 mul_prime(uint32_t s) const { Kb4 r; for (int i = 0; i < 4; ++i) r.c[i] = kb_mul(c[i], s); return r; }

  // x -> x^(p^power): coefficient i times phase^i, phase = [1, 2113994754,
  // 2130706432, 16711679][power mod 4] (koalabear.rs frobenius).
  Kb4 frobenius(int power) const {
    static const uint32_t phases[4] = {1u, 2113994754u, 2130706432u, 16711679u};
    power %= 4;
    if (power < 0) power += 4;
    const uint32_t phase = phases[power];
    Kb4 r;
    uint32_t scale = 1;
    for (int i = 0; i < 4; ++i) {
      r.c[i] = kb_mul(c[i], scale);
      scale = kb_mul(scale, phase);
    }
    return r;
  }
  // Inverse through the norm: x^-1 = (x^p * x^(p^2) * x^(p^3)) / N(x).
  bool try_inverse(Kb4& out) const {
    if (is_zero()) return false;
    Kb4 prod = frobenius(1);
    for (int k = 2; k < 4; ++k) prod = (prod * *this).frobenius(1);
    Kb4 norm = *this * prod;
    out = prod.mul_prime(kb_inv(norm.c[0]));
    return true;
  }
  Kb4 inverse() const { Kb4 r; try_inverse(r); return r; }

  static constexpr int kBytes = 16;
  QF_HD void to_bytes(uint8_t out[16]) const {
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) out[4 * i + j] = uint8_t(c[i] >> (8 * j));
  }
  static bool from_bytes(const uint8_t in[16], Kb4& out) {
    for (int i = 0; i < 4; ++i) {
      uint32_t v = 0;
      for (int j = 0; j < 4; ++j) v |= uint32_t(in[4 * i + j]) << (8 * j);
      if (v >= PKB) return false;
      out.c[i] = v;
    }
    return true;
  }
  // Uniform sampling drops the top bit of each little-endian word, then
  // rejects words >= p.
  static bool from_uniform_bytes(const uint8_t in[16], Kb4& out) {
    uint8_t b[16];
    std::memcpy(b, in, 16);
    for (int i : {3, 7, 11, 15}) b[i] &= 0x7f;
    return from_bytes(b, out);
  }
  // Signed small integer embedding into coefficient zero (field.rs:25-29).
  QF_HD static uint32_t small(int v) { int64_t r = int64_t(v) % int64_t(PKB); return uint32_t(r < 0 ? r + PKB : r); }
  static uint64_t modulus_u64() { return PKB; }
};

}  // namespace qf
