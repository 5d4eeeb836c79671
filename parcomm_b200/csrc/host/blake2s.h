// BLAKE2s-256 (RFC 7693), unkeyed, 32-byte digest, streaming with copyable state.
//
// The reference hashes with the `blake2` 0.10 crate (Blake2s256) and with
// `blake2s_simd` 0.5.4 `hash_many`; both are plain BLAKE2s-256 with default
// parameters (qafold/f65521/vendor/qafold/Cargo.toml:15-16).  Running
// transcripts clone a partially absorbed state before finalising a challenge
// (qafold_short_pc.rs:2186-2197), so the state here is a value type.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
#include <immintrin.h>
#endif
#include <array>
#include <string>
#include <vector>

namespace qf {

using Digest = std::array<uint8_t, 32>;

static constexpr uint32_t kBlake2sIv[8] = {
    0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
    0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};

static constexpr uint8_t kBlake2sSigma[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
    {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4},
    {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13},
    {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11},
    {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5},
    {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};

inline uint32_t rotr32(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
// The same compression with the four columns of the state in SSE registers
// (the rows of RFC 7693's 4 x 4 matrix, diagonalised by lane rotations
// between the column and diagonal steps; rotations by 16 and 8 as byte
// shuffles).  Compiled for SSSE3 and chosen at run time.
__attribute__((target("ssse3"))) inline void blake2s_compress_ssse3(uint32_t h[8], const uint8_t block[64], uint64_t t,
                                                                    bool last) {
  uint32_t m[16];
  std::memcpy(m, block, 64);  // little-endian words
  const __m128i r16 = _mm_setr_epi8(2, 3, 0, 1, 6, 7, 4, 5, 10, 11, 8, 9, 14, 15, 12, 13);
  const __m128i r8 = _mm_setr_epi8(1, 2, 3, 0, 5, 6, 7, 4, 9, 10, 11, 8, 13, 14, 15, 12);
  __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(h));
  __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(h + 4));
  const __m128i a0 = a, b0 = b;
  __m128i c = _mm_setr_epi32(int(kBlake2sIv[0]), int(kBlake2sIv[1]), int(kBlake2sIv[2]), int(kBlake2sIv[3]));
  __m128i d = _mm_xor_si128(_mm_setr_epi32(int(kBlake2sIv[4]), int(kBlake2sIv[5]), int(kBlake2sIv[6]), int(kBlake2sIv[7])),
                            _mm_setr_epi32(int(uint32_t(t)), int(uint32_t(t >> 32)), last ? -1 : 0, 0));
#define QF_G4(x, y)                                                                            \
  a = _mm_add_epi32(_mm_add_epi32(a, b), x);                                                   \
  d = _mm_shuffle_epi8(_mm_xor_si128(d, a), r16);                                              \
  c = _mm_add_epi32(c, d);                                                                     \
  b = _mm_xor_si128(b, c);                                                                     \
  b = _mm_or_si128(_mm_srli_epi32(b, 12), _mm_slli_epi32(b, 20));                              \
  a = _mm_add_epi32(_mm_add_epi32(a, b), y);                                                   \
  d = _mm_shuffle_epi8(_mm_xor_si128(d, a), r8);                                               \
  c = _mm_add_epi32(c, d);                                                                     \
  b = _mm_xor_si128(b, c);                                                                     \
  b = _mm_or_si128(_mm_srli_epi32(b, 7), _mm_slli_epi32(b, 25));
#pragma GCC unroll 10
  for (int r = 0; r < 10; ++r) {
    const uint8_t* s = kBlake2sSigma[r];
    QF_G4(_mm_setr_epi32(int(m[s[0]]), int(m[s[2]]), int(m[s[4]]), int(m[s[6]])),
          _mm_setr_epi32(int(m[s[1]]), int(m[s[3]]), int(m[s[5]]), int(m[s[7]])));
    b = _mm_shuffle_epi32(b, _MM_SHUFFLE(0, 3, 2, 1));  // lanes: (v0, v5, v10, v15), ...
    c = _mm_shuffle_epi32(c, _MM_SHUFFLE(1, 0, 3, 2));
    d = _mm_shuffle_epi32(d, _MM_SHUFFLE(2, 1, 0, 3));
    QF_G4(_mm_setr_epi32(int(m[s[8]]), int(m[s[10]]), int(m[s[12]]), int(m[s[14]])),
          _mm_setr_epi32(int(m[s[9]]), int(m[s[11]]), int(m[s[13]]), int(m[s[15]])));
    b = _mm_shuffle_epi32(b, _MM_SHUFFLE(2, 1, 0, 3));
    c = _mm_shuffle_epi32(c, _MM_SHUFFLE(1, 0, 3, 2));
    d = _mm_shuffle_epi32(d, _MM_SHUFFLE(0, 3, 2, 1));
  }
#undef QF_G4
  _mm_storeu_si128(reinterpret_cast<__m128i*>(h), _mm_xor_si128(a0, _mm_xor_si128(a, c)));
  _mm_storeu_si128(reinterpret_cast<__m128i*>(h + 4), _mm_xor_si128(b0, _mm_xor_si128(b, d)));
}
#endif

// One compression of a 64-byte block.  `t` is the byte counter after this
// block, `last` marks the final block.
inline void blake2s_compress_scalar(uint32_t h[8], const uint8_t block[64], uint64_t t, bool last) {
  uint32_t m[16];
  for (int i = 0; i < 16; ++i) {
    m[i] = uint32_t(block[4 * i]) | (uint32_t(block[4 * i + 1]) << 8) |
           (uint32_t(block[4 * i + 2]) << 16) | (uint32_t(block[4 * i + 3]) << 24);
  }
  uint32_t v[16];
  for (int i = 0; i < 8; ++i) { v[i] = h[i]; v[i + 8] = kBlake2sIv[i]; }
  v[12] ^= uint32_t(t);
  v[13] ^= uint32_t(t >> 32);
  if (last) v[14] = ~v[14];
#define QF_G(a, b, c, d, x, y)        \
  v[a] = v[a] + v[b] + x;             \
  v[d] = rotr32(v[d] ^ v[a], 16);     \
  v[c] = v[c] + v[d];                 \
  v[b] = rotr32(v[b] ^ v[c], 12);     \
  v[a] = v[a] + v[b] + y;             \
  v[d] = rotr32(v[d] ^ v[a], 8);      \
  v[c] = v[c] + v[d];                 \
  v[b] = rotr32(v[b] ^ v[c], 7);
  // Unrolled, the schedule's indices are constants and m[] stays in registers.
#pragma GCC unroll 10
  for (int r = 0; r < 10; ++r) {
    const uint8_t* s = kBlake2sSigma[r];
    QF_G(0, 4, 8, 12, m[s[0]], m[s[1]]);
    QF_G(1, 5, 9, 13, m[s[2]], m[s[3]]);
    QF_G(2, 6, 10, 14, m[s[4]], m[s[5]]);
    QF_G(3, 7, 11, 15, m[s[6]], m[s[7]]);
    QF_G(0, 5, 10, 15, m[s[8]], m[s[9]]);
    QF_G(1, 6, 11, 12, m[s[10]], m[s[11]]);
    QF_G(2, 7, 8, 13, m[s[12]], m[s[13]]);
    QF_G(3, 4, 9, 14, m[s[14]], m[s[15]]);
  }
#undef QF_G
  for (int i = 0; i < 8; ++i) h[i] ^= v[i] ^ v[i + 8];
}

inline void blake2s_compress(uint32_t h[8], const uint8_t block[64], uint64_t t, bool last) {
#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
  static const bool ssse3 = __builtin_cpu_supports("ssse3");
  if (ssse3) {
    blake2s_compress_ssse3(h, block, t, last);
    return;
  }
#endif
  blake2s_compress_scalar(h, block, t, last);
}

class Blake2s {
 public:
  Blake2s() {
    for (int i = 0; i < 8; ++i) h_[i] = kBlake2sIv[i];
    h_[0] ^= 0x01010000u ^ 32u;  // digest length 32, no key, fanout 1, depth 1
  }
  void update(const void* data, size_t len) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    while (len > 0) {
      if (buflen_ == 64) {  // a full buffer is compressed only once more input arrives
        t_ += 64;
        blake2s_compress(h_, buf_, t_, false);
        buflen_ = 0;
      }
      // Whole blocks straight from the input while more input follows them.
      while (buflen_ == 0 && len > 64) {
        t_ += 64;
        blake2s_compress(h_, p, t_, false);
        p += 64;
        len -= 64;
      }
      size_t take = 64 - buflen_;
      if (take > len) take = len;
      std::memcpy(buf_ + buflen_, p, take);
      buflen_ += take;
      p += take;
      len -= take;
    }
  }
  void update(const std::vector<uint8_t>& v) { update(v.data(), v.size()); }
  void update(const Digest& d) { update(d.data(), d.size()); }
  void update_str(const char* s) { update(s, std::strlen(s)); }
  void update_u64(uint64_t x) {
    uint8_t b[8];
    for (int i = 0; i < 8; ++i) b[i] = uint8_t(x >> (8 * i));
    update(b, 8);
  }
  Digest finalize() const {
    uint32_t h[8];
    std::memcpy(h, h_, sizeof(h));
    uint8_t block[64];
    std::memset(block, 0, 64);
    std::memcpy(block, buf_, buflen_);
    blake2s_compress(h, block, t_ + buflen_, true);
    Digest out;
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 4; ++j) out[4 * i + j] = uint8_t(h[i] >> (8 * j));
    return out;
  }
  // Chaining value and counter after absorbing exactly `n` whole 64-byte
  // blocks that are known not to be the last (midstate for device hashing).
  void midstate(uint32_t h_out[8]) const { std::memcpy(h_out, h_, sizeof(h_)); }
  uint64_t counter() const { return t_; }
  size_t buffered() const { return buflen_; }

 private:
  uint32_t h_[8];
  uint64_t t_ = 0;
  uint8_t buf_[64];
  size_t buflen_ = 0;
};

inline Digest blake2s(const void* data, size_t len) {
  Blake2s h;
  h.update(data, len);
  return h.finalize();
}

// Framing used by every reference hash domain: u64le(len(label)) || label ||
// u64le(len(bytes)) || bytes  (qafold_short_pc.rs:2178-2183).
inline void absorb_framed(Blake2s& h, const char* label, const void* bytes, size_t len) {
  size_t ll = std::strlen(label);
  h.update_u64(ll);
  h.update(label, ll);
  h.update_u64(len);
  h.update(bytes, len);
}
inline void absorb_framed_u64(Blake2s& h, const char* label, uint64_t v) {
  uint8_t b[8];
  for (int i = 0; i < 8; ++i) b[i] = uint8_t(v >> (8 * i));
  absorb_framed(h, label, b, 8);
}
inline void append_frame(std::vector<uint8_t>& out, const char* label, const void* bytes, size_t len) {
  size_t ll = std::strlen(label);
  for (int i = 0; i < 8; ++i) out.push_back(uint8_t(uint64_t(ll) >> (8 * i)));
  out.insert(out.end(), label, label + ll);
  for (int i = 0; i < 8; ++i) out.push_back(uint8_t(uint64_t(len) >> (8 * i)));
  const uint8_t* p = static_cast<const uint8_t*>(bytes);
  out.insert(out.end(), p, p + len);
}
inline void put_u64(std::vector<uint8_t>& out, uint64_t v) {
  for (int i = 0; i < 8; ++i) out.push_back(uint8_t(v >> (8 * i)));
}
inline std::array<uint8_t, 8> le64(uint64_t v) {
  std::array<uint8_t, 8> b;
  for (int i = 0; i < 8; ++i) b[i] = uint8_t(v >> (8 * i));
  return b;
}
inline std::string hex(const uint8_t* p, size_t n) {
  static const char* d = "0123456789abcdef";
  std::string s;
  for (size_t i = 0; i < n; ++i) { s.push_back(d[p[i] >> 4]); s.push_back(d[p[i] & 15]); }
  return s;
}
inline std::string hex(const Digest& d) { return hex(d.data(), d.size()); }

}  // namespace qf
