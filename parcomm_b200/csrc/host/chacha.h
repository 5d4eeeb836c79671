// `rand` 0.8 StdRng: ChaCha12 with a 64-bit block counter and a zero stream
// id (rand_chacha 0.3.1), buffered four blocks at a time as in rand_core
// 0.6.4's BlockRng.  The reference draws the QAFold setup seed with
// `StdRng::from_seed([0x51; 32]).fill_bytes(&mut [0u8; 32])`
// (packed.rs:134-158, qafold_short_pc.rs:401-406); its wire fixture test uses
// `StdRng::seed_from_u64` and `sample_uniform` (qafold_short_pc.rs:3605-3614).
#pragma once
#include <cstdint>
#include <cstring>
#include <array>

namespace qf {

class StdRng {
 public:
  explicit StdRng(const std::array<uint8_t, 32>& seed) {
    for (int i = 0; i < 8; ++i)
      key_[i] = uint32_t(seed[4 * i]) | (uint32_t(seed[4 * i + 1]) << 8) |
                (uint32_t(seed[4 * i + 2]) << 16) | (uint32_t(seed[4 * i + 3]) << 24);
    index_ = 64;
  }
  // rand_core 0.6 `SeedableRng::seed_from_u64`: PCG32 output words fill the seed.
  static StdRng seed_from_u64(uint64_t state) {
    std::array<uint8_t, 32> seed{};
    for (int chunk = 0; chunk < 8; ++chunk) {
      state = state * 6364136223846793005ull + 11634580027462260723ull;
      uint32_t xorshifted = uint32_t(((state >> 18) ^ state) >> 27);
      uint32_t rot = uint32_t(state >> 59);
      uint32_t x = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
      for (int j = 0; j < 4; ++j) seed[4 * chunk + j] = uint8_t(x >> (8 * j));
    }
    return StdRng(seed);
  }
  uint32_t next_u32() {
    if (index_ >= 64) generate(), index_ = 0;
    return results_[index_++];
  }
  uint64_t next_u64() {
    if (index_ < 63) {
      uint64_t lo = results_[index_], hi = results_[index_ + 1];
      index_ += 2;
      return lo | (hi << 32);
    }
    if (index_ >= 64) {
      generate();
      index_ = 2;
      return uint64_t(results_[0]) | (uint64_t(results_[1]) << 32);
    }
    uint64_t x = results_[63];
    generate();
    index_ = 1;
    return x | (uint64_t(results_[0]) << 32);
  }
  void fill_bytes(uint8_t* dest, size_t len) {
    size_t read = 0;
    while (read < len) {
      if (index_ >= 64) generate(), index_ = 0;
      // Consume whole words; a partial final word is still consumed entirely.
      size_t avail_words = 64 - index_;
      size_t want = len - read;
      size_t words = (want + 3) / 4;
      if (words > avail_words) words = avail_words;
      size_t bytes = words * 4 < want ? words * 4 : want;
      uint8_t tmp[256];
      for (size_t w = 0; w < words; ++w)
        for (int j = 0; j < 4; ++j) tmp[4 * w + j] = uint8_t(results_[index_ + w] >> (8 * j));
      std::memcpy(dest + read, tmp, bytes);
      index_ += words;
      read += bytes;
    }
  }

 private:
  static uint32_t rotl(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }
  void generate() {
    for (int b = 0; b < 4; ++b) {
      uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
      for (int i = 0; i < 8; ++i) s[4 + i] = key_[i];
      s[12] = uint32_t(counter_);
      s[13] = uint32_t(counter_ >> 32);
      s[14] = 0;
      s[15] = 0;
      uint32_t x[16];
      std::memcpy(x, s, sizeof(x));
#define QF_QR(a, b, c, d)                 \
  x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 16); \
  x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 12); \
  x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 8);  \
  x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 7);
      for (int r = 0; r < 6; ++r) {  // 12 rounds = 6 double rounds
        QF_QR(0, 4, 8, 12); QF_QR(1, 5, 9, 13); QF_QR(2, 6, 10, 14); QF_QR(3, 7, 11, 15);
        QF_QR(0, 5, 10, 15); QF_QR(1, 6, 11, 12); QF_QR(2, 7, 8, 13); QF_QR(3, 4, 9, 14);
      }
#undef QF_QR
      for (int i = 0; i < 16; ++i) results_[16 * b + i] = x[i] + s[i];
      ++counter_;
    }
  }
  uint32_t key_[8];
  uint64_t counter_ = 0;
  uint32_t results_[64];
  size_t index_;
};

}  // namespace qf
