// F_65521 and the octic field F_65521[X]/(X^8 - 17), used directly as the
// QAFold message field for 8-bit weights.
//
// Reference: Prime65521 (qafold_short.rs:325-480, `reduce_u32` 336-346),
// Prime65521Ext8 (qafold_short.rs:482-660: Frobenius root 57852 at 486-495,
// `mul_add` 515-525, `try_inverse` 628-640) and FullPrime65521Ext8
// (full_extension.rs:21-214: canonical 16-byte encoding, NAME, uniform
// sampling by canonical rejection).  Arithmetic is exact, so any correct
// reduction order gives identical canonical results.
#pragma once
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define QF_HD __host__ __device__ __forceinline__
#else
#define QF_HD inline
#endif

namespace qf {

static constexpr uint32_t P65521 = 65521u;

QF_HD uint32_t fp_reduce32(uint32_t v) {  // v < 2^32 -> canonical
  uint32_t f = (v & 0xffffu) + 15u * (v >> 16);
  f = (f & 0xffffu) + 15u * (f >> 16);
  return f >= P65521 ? f - P65521 : f;
}
QF_HD uint32_t fp_reduce64(uint64_t v) {  // v < 2^48 -> canonical
  uint64_t f = (v & 0xffffu) + 15u * (v >> 16);  // < 2^36
  f = (f & 0xffffu) + 15u * (f >> 16);           // < 2^24
  return fp_reduce32(uint32_t(f));
}
QF_HD uint32_t fp_add(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P65521 ? s - P65521 : s; }
QF_HD uint32_t fp_sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P65521 - b; }
QF_HD uint32_t fp_mul(uint32_t a, uint32_t b) { return fp_reduce32(a * b); }
QF_HD uint32_t fp_neg(uint32_t a) { return a == 0 ? 0 : P65521 - a; }
inline uint32_t fp_pow(uint32_t a, uint64_t e) {
  uint32_t r = 1;
  while (e) { if (e & 1) r = fp_mul(r, a); a = fp_mul(a, a); e >>= 1; }
  return r;
}
inline uint32_t fp_inv(uint32_t a) { return fp_pow(a, P65521 - 2); }

// omega = 17^((p-1)/8) = 57852; Frobenius multiplies coefficient i by omega^i.
static constexpr uint16_t kFrobRoot[8] = {1, 57852, 0, 0, 0, 0, 0, 0};

struct Fp8 {
  using Coeff = uint16_t;
  uint16_t c[8];
  // Packed-PCS transcript domain and single-block proof magic (packed.rs:19, 442).
  static constexpr const char* kPackedDomain = "mikros/qafold-f65521-ext8/packed-boolean-mle/v1";
  static constexpr const char* kPackedMagic = "QA655PK1";
  // Outer protocol transcript and opening-context domains (transcript.rs:15, protocol.rs:323).
  static constexpr const char* kPublicDomain = "parcomm-qafold/public/v1";
  static constexpr const char* kTerminalDomain = "parcomm/qafold/terminal/v2";
  static uint32_t base_mul(uint32_t a, uint32_t b) { return fp_mul(a, b); }
  static uint32_t base_inv(uint32_t a) { return fp_inv(a % P65521); }
  // The primitive 8th root of unity 17^((p-1)/8) used by the lane DFT, inverted.
  static uint32_t root_of_unity_inverse() { return fp_inv(57852u); }

  static constexpr int kLanes = 8;          // base values packed per element
  static constexpr uint32_t kPrime = P65521;
  static constexpr const char* kName = "FullPrime65521Ext8/X^8-17/v1";
  // Field cardinality p^8 as the integer the reference converts to f64.
  static unsigned __int128 cardinality() {
    unsigned __int128 r = 1;
    for (int i = 0; i < 8; ++i) r *= P65521;
    return r;
  }

  QF_HD static Fp8 zero() { Fp8 r; for (int i = 0; i < 8; ++i) r.c[i] = 0; return r; }
  QF_HD static Fp8 one() { Fp8 r = zero(); r.c[0] = 1; return r; }
  QF_HD static Fp8 from_base(uint32_t v) { Fp8 r = zero(); r.c[0] = uint16_t(v); return r; }
  QF_HD bool is_zero() const { for (int i = 0; i < 8; ++i) if (c[i]) return false; return true; }
  QF_HD bool operator==(const Fp8& o) const { for (int i = 0; i < 8; ++i) if (c[i] != o.c[i]) return false; return true; }
  QF_HD bool operator!=(const Fp8& o) const { return !(*this == o); }
  QF_HD Fp8 operator+(const Fp8& o) const { Fp8 r; for (int i = 0; i < 8; ++i) r.c[i] = uint16_t(fp_add(c[i], o.c[i])); return r; }
  QF_HD Fp8 operator-(const Fp8& o) const { Fp8 r; for (int i = 0; i < 8; ++i) r.c[i] = uint16_t(fp_sub(c[i], o.c[i])); return r; }
  QF_HD Fp8 operator-() const { Fp8 r; for (int i = 0; i < 8; ++i) r.c[i] = uint16_t(fp_neg(c[i])); return r; }
  QF_HD Fp8& operator+=(const Fp8& o) { *this = *this + o; return *this; }
  QF_HD Fp8& operator-=(const Fp8& o) { *this = *this - o; return *this; }
  QF_HD Fp8 operator*(const Fp8& o) const {
    // Schoolbook product with X^8 = 17; each accumulator < 8*17*65520^2 < 2^40.
    uint64_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 8; ++i) {
      uint64_t a = c[i];
      for (int j = 0; j < 8; ++j) {
        uint64_t p = a * o.c[j];
        int k = i + j;
        if (k < 8) acc[k] += p; else acc[k - 8] += 17u * p;
      }
    }
    Fp8 r;
    for (int k = 0; k < 8; ++k) r.c[k] = uint16_t(fp_reduce64(acc[k]));
    return r;
  }
  QF_HD Fp8& operator*=(const Fp8& o) { *this = *this * o; return *this; }
  QF_HD Fp8 mul_prime(uint32_t s) const { Fp8 r; for (int i = 0; i < 8; ++i) r.c[i] = uint16_t(fp_mul(c[i], s)); return r; }

  // x -> x^(p^power): coefficient i times omega^(i*power mod 8).
  Fp8 frobenius(int power) const {
    static const uint32_t roots[8] = {1u, 57852u, fp_mul(57852u, 57852u),
                                      fp_mul(fp_mul(57852u, 57852u), 57852u), P65521 - 1,
                                      fp_mul(P65521 - 1, 57852u),
                                      fp_mul(P65521 - 1, fp_mul(57852u, 57852u)),
                                      fp_mul(P65521 - 1, fp_mul(fp_mul(57852u, 57852u), 57852u))};
    power %= 8;
    if (power < 0) power += 8;
    Fp8 r;
    for (int i = 0; i < 8; ++i) r.c[i] = uint16_t(fp_mul(c[i], roots[(i * power) % 8]));
    return r;
  }
  // Inverse through the norm: x^-1 = (x^p * ... * x^(p^7)) / N(x).
  bool try_inverse(Fp8& out) const {
    if (is_zero()) return false;
    Fp8 prod = frobenius(1);
    for (int k = 2; k < 8; ++k) prod = (prod * *this).frobenius(1);
    Fp8 norm = *this * prod;
    out = prod.mul_prime(fp_inv(norm.c[0]));
    return true;
  }
  Fp8 inverse() const { Fp8 r; try_inverse(r); return r; }

  static constexpr int kBytes = 16;
  QF_HD void to_bytes(uint8_t out[16]) const {
    for (int i = 0; i < 8; ++i) { out[2 * i] = uint8_t(c[i]); out[2 * i + 1] = uint8_t(c[i] >> 8); }
  }
  static bool from_bytes(const uint8_t in[16], Fp8& out) {
    for (int i = 0; i < 8; ++i) {
      uint32_t v = uint32_t(in[2 * i]) | (uint32_t(in[2 * i + 1]) << 8);
      if (v >= P65521) return false;
      out.c[i] = uint16_t(v);
    }
    return true;
  }
  // Uniform sampling accepts a 16-byte string iff it is canonical
  // (full_extension.rs:175-180).
  static bool from_uniform_bytes(const uint8_t in[16], Fp8& out) { return from_bytes(in, out); }
  // Signed small integer embedding into coefficient zero (field.rs:24-29).
  QF_HD static uint32_t small(int v) { int r = v % int(P65521); return uint32_t(r < 0 ? r + int(P65521) : r); }
  // Canonical base modulus bytes (8-byte LE, the short-field framing).
  static uint64_t modulus_u64() { return P65521; }
};

}  // namespace qf
