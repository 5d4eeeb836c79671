// Constant BLAKE2s prefixes of the row-leaf and inner-node messages, computed
// on the host and passed to the hashing kernels by value.
#pragma once
#include <cstdint>

namespace qfd {

// Leaf message = 75-byte prefix (framed domain and width) || row bytes.  The
// first 64 bytes are absorbed into `mid`; `tail` holds prefix bytes 64..74.
struct LeafPrefix {
  uint32_t mid[8];
  uint32_t tail[3];
};

// Inner message = 50-byte framed domain || left || right.
struct InnerPrefix {
  uint32_t w[13];  // last word holds 2 bytes
};

}  // namespace qfd
