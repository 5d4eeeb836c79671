// Constant BLAKE2s prefixes of the row-leaf and inner-node messages, computed
// on the host and passed to the hashing kernels by value.
#pragma once
#include <cstdint>

namespace qfd {

// Leaf message = prefix (framed domain and width; 75 bytes for base rows,
// 80 for extension rows) || row bytes.  The first 64 bytes are absorbed into
// `mid`; `tail` holds the remaining prefix bytes.
struct LeafPrefix {
  uint32_t mid[8];
  uint32_t tail[4];  // 11 (base-row) or 16 (extension-row) bytes
  uint32_t one = 1;  // the multiplier of the compression's multiply-add additions
};

// Setup-row leaf message = constant framed prefix || framed row index ||
// row bytes.  The prefix's first t0 bytes (whole blocks) are absorbed into
// `mid`; `tail` holds the n_tail (1..64) bytes after them.
struct SetupLeafPrefix {
  uint32_t mid[8];
  uint32_t t0;
  uint32_t n_tail;
  uint32_t tail[16];
  uint32_t one = 1;  // the multiplier of the compression's multiply-add additions
};

// Inner message = 50-byte framed domain || left || right.
struct InnerPrefix {
  uint32_t w[13];  // last word holds 2 bytes
  uint32_t one = 1;  // the multiplier of the compression's multiply-add additions
};

}  // namespace qfd
