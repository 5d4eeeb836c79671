// Field-independent CUDA infrastructure of the library: error checks, the
// per-kernel timer, the device memory pool, device buffers, launch sizing and
// the constant BLAKE2s prefixes of the Merkle hashing.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "device/hash_prefix.h"
#include "host/protocol.h"
#include "host/sections.h"

namespace qfg {
using namespace qf;

#define QF_CK(x)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (x);                                                                     \
    if (e_ != cudaSuccess)                                                                    \
      ::qf::fail(QF_E_CUDA, std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #x); \
  } while (0)

// Process-wide kernel choices, for comparisons that must write the same
// bytes: `imma` runs the F65521 weight passes on the tensor cores (exact
// integer limbs) instead of the dp4a / IMAD kernels (off by default: slower
// as measured on B200); `per_matrix` issues the
// weight passes one launch per term, bucket or block instead of one launch
// over all of them; `core_dots` chooses where the extension-product sums of
// the EO, sumcheck and LiteBullet rounds run: 0 (default) per kernel as
// measured fastest, 1 all on the CUDA cores, 2 all on the tensor cores.  Set
// through qf_kernel_option.
struct KernelOptions {
  static std::atomic<int> imma;
  static std::atomic<int> per_matrix;
  static std::atomic<int> core_dots;
};

// Per-kernel device time: when enabled, every launch is bracketed by CUDA
// events recorded on the launching stream; totals are read after a sync.
struct KernelClock {
  struct Rec { const char* name; cudaEvent_t a, b; uint64_t bytes, ops; };
  struct Scope {
    cudaStream_t stream;
    const char* name;
    uint64_t bytes;  // algorithmic bytes moved by this launch
    uint64_t ops;    // algorithmic integer operations (thread level) of this launch, 0 if not counted
    cudaEvent_t a = nullptr, b = nullptr;
    Scope(cudaStream_t s, const char* n, uint64_t bytes, uint64_t ops = 0);
    void done();
  };
  static bool enabled;
  static std::mutex mu;
  static std::vector<Rec> recs;
  static std::atomic<uint64_t> launches;
  static void reset(bool on);
  static std::string stats_json();
  // A named JSON value reported under "_notes" in stats_json (tuning results).
  static void note(const std::string& key, const std::string& json_value);
};

// Host wall time of named sections (recorded while KernelClock is enabled).
using HostScope = ::qf::Section;

#define QF_LAUNCH(stream, name, bytes, ...)     \
  do {                                          \
    ::qfg::KernelClock::Scope qf_scope_(stream, name, bytes); \
    __VA_ARGS__;                                \
    QF_CK(cudaGetLastError());                  \
    qf_scope_.done();                           \
  } while (0)
// The same, with the launch's algorithmic integer operations (intops.h).
#define QF_LAUNCH_OPS(stream, name, bytes, ops, ...)     \
  do {                                                   \
    ::qfg::KernelClock::Scope qf_scope_(stream, name, bytes, ops); \
    __VA_ARGS__;                                         \
    QF_CK(cudaGetLastError());                           \
    qf_scope_.done();                                    \
  } while (0)

// Process-wide cache of device allocations: released buffers are kept, keyed
// by device and rounded size, and handed out again, so repeated commits/openings
// of the same shapes pay no cudaMalloc/cudaFree.  A failed cudaMalloc frees
// cached blocks, largest first, until the request fits.
struct DevicePool {
  static void* get(size_t bytes);
  static void put(void* p, size_t bytes);
  static void trim();
  static bool evict_one();  // frees the largest cached block of the current device
  static size_t cached_bytes();  // held in the cache for the current device
  // At most `bytes` stay cached (all devices); further released blocks are
  // freed at once.  Unlimited by default.
  static void set_limit(size_t bytes);
  static size_t rounded(size_t bytes) {
    const size_t g = bytes >= (size_t(1) << 20) ? (size_t(1) << 20) : 256;
    return (bytes + g - 1) / g * g;
  }
};

// A process-wide page-locked host buffer for device-to-host copies of proof
// payloads: a copy into it runs at link speed, where one into pageable memory
// is staged by the driver.  One holder at a time (the lease keeps a lock);
// it grows to the largest request and is portable across devices.
struct PinnedStage {
  struct Lease {
    std::unique_lock<std::mutex> lock;
    void* p = nullptr;
  };
  static Lease acquire(size_t bytes);
};

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept { reset(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; return *this; }
  ~DBuf() { reset(); }
  void alloc(size_t count) {
    reset();
    if (count) p = static_cast<T*>(DevicePool::get(count * sizeof(T)));
    n = count;
  }
  void reset() {
    if (p) DevicePool::put(p, n * sizeof(T));
    p = nullptr;
    n = 0;
  }
};

inline int grid_for(uint64_t n, int threads, int max_blocks = 148 * 8) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > uint64_t(max_blocks)) b = max_blocks;
  return int(b);
}

// Constant hash prefixes computed on the host.
qfd::LeafPrefix leaf_prefix(size_t n_cols, bool ext_domain);
qfd::InnerPrefix inner_prefix();

// A digest held as two uint4 words (the Merkle tree layout in device memory).
inline Digest digest_from_words(const uint4* d) {
  Digest out;
  uint32_t w[8] = {d[0].x, d[0].y, d[0].z, d[0].w, d[1].x, d[1].y, d[1].z, d[1].w};
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 4; ++j) out[4 * i + j] = uint8_t(w[i] >> (8 * j));
  return out;
}

}  // namespace qfg
