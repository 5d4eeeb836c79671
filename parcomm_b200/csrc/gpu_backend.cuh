// CUDA implementation of the packed-PCS / EO backend for F65521^8 with int8
// weights.  All bulk data (BVA, codewords, Merkle trees, EO and sumcheck
// vectors) stays in HBM; only transcript-sized values cross to the host.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "host/protocol.h"
#include "host/sections.h"
#include "device/f65521_dev.cuh"
#include "device/hash_prefix.h"

namespace qfg {
using namespace qf;
using F = Fp8;
using qfd::Fe;

#define QF_CK(x)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (x);                                                                     \
    if (e_ != cudaSuccess)                                                                    \
      ::qf::fail(QF_E_CUDA, std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #x); \
  } while (0)

// Per-kernel device time: when enabled, every launch is bracketed by CUDA
// events recorded on the launching stream; totals are read after a sync.
struct KernelClock {
  struct Rec { const char* name; cudaEvent_t a, b; uint64_t bytes; };
  struct Scope {
    cudaStream_t stream;
    const char* name;
    uint64_t bytes;  // algorithmic bytes moved by this launch
    cudaEvent_t a = nullptr, b = nullptr;
    Scope(cudaStream_t s, const char* n, uint64_t bytes);
    void done();
  };
  static bool enabled;
  static std::mutex mu;
  static std::vector<Rec> recs;
  static std::atomic<uint64_t> launches;
  static void reset(bool on);
  static std::string stats_json();
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

// Process-wide cache of device allocations: released buffers are kept, keyed
// by their rounded size, and handed out again, so repeated commits/openings
// of the same shapes pay no cudaMalloc/cudaFree.  A failed cudaMalloc first
// returns the cache to the driver and retries.
struct DevicePool {
  static void* get(size_t bytes);
  static void put(void* p, size_t bytes);
  static void trim();
  static size_t rounded(size_t bytes) {
    const size_t g = bytes >= (size_t(1) << 20) ? (size_t(1) << 20) : 256;
    return (bytes + g - 1) / g * g;
  }
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

inline const Fe* as_fe(const F* p) { return reinterpret_cast<const Fe*>(p); }
inline Fe to_fe(const F& v) { Fe e; std::memcpy(&e, &v, 16); return e; }
inline F from_fe(const Fe& e) { F v; std::memcpy(&v, &e, 16); return v; }

inline int grid_for(uint64_t n, int threads, int max_blocks = 148 * 8) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > uint64_t(max_blocks)) b = max_blocks;
  return int(b);
}

// Device copies of a parameter set's code alphas (alphas[0] and alphas[1] of
// every level), uploaded once per device and shared by every commitment and
// opening made with that parameter set.  Thread-safe; an upload completes
// before the pointer is returned, so any stream may read it.
class DeviceTables {
 public:
  const Fe* alpha(const PcsParams<F>& pp, size_t level, int which);
  const Fe* top_alpha1(const PcsParams<F>& pp) { return alpha(pp, pp.seq.codes.size() - 1, 1); }

 private:
  std::mutex mu_;
  std::map<std::tuple<int, size_t, int>, DBuf<Fe>> bufs_;  // (device, level, which)
};

// Constant hash prefixes computed on the host.
qfd::LeafPrefix leaf_prefix(size_t n_cols, bool ext_domain);
qfd::InnerPrefix inner_prefix();

// A committed codeword in HBM: column-major entries and all Merkle levels.
struct DeviceCodeword : CodewordView<F> {
  cudaStream_t stream = nullptr;
  DBuf<Fe> cw;          // n_cols x n_ext
  DBuf<uint4> tree;     // 2 uint4 per digest, levels concatenated (leaves first)
  std::vector<uint64_t> level_off;
  size_t n_ext = 0, n_cols = 0;
  Digest root_{};

  Digest root() const override { return root_; }
  size_t ext_rows() const override { return n_ext; }
  size_t cols() const override { return n_cols; }
  std::vector<F> fold_rows(size_t n_rows, const std::vector<F>& w) const override;
  std::vector<F> project_rows(size_t n_rows, const std::vector<F>& w) const override;
  std::vector<std::vector<F>> rows(const std::vector<size_t>& idx) const override;
  std::vector<std::vector<Digest>> paths(const std::vector<size_t>& idx) const override;
  std::vector<F> entries() const override;
};

// Commitment root of block `b` of a device BVA (`active` entries), computed
// only in the caller's device buffers: `cw` holds 2R x cols entries, `tree`
// 4 x 2R words (2 x 2R digests), `alpha` R entries (overwritten with the
// code's alpha table).  Launches on `s`, writes the 32-byte root to the device
// bytes `d_root` and returns without synchronising; allocates no device memory.
void commit_block_into(const Parameters<F>& P, const int8_t* d_bva, uint64_t active, size_t b, Fe* cw, uint4* tree,
                       Fe* alpha, uint8_t* d_root, cudaStream_t s);

class GpuBackend : public Backend<F>,
                   public SingleBackend<F>,
                   public EoBackend<F>,
                   public TopRoundAccel<F>,
                   public DecideAccel<F> {
 public:
  // `tables` (optional, not owned) shares uploaded code tables across backends.
  GpuBackend(const Parameters<F>& p, const int8_t* d_bva, size_t active, cudaStream_t s, DeviceTables* tables = nullptr);
  ~GpuBackend() override;

  // commit
  Digest commit_block(size_t b) override;
  Digest commit() override { return commit_block(0); }
  const std::vector<Digest>& roots() const { return roots_; }

  // batch opening
  std::vector<std::vector<F>> project_blocks(const std::vector<F>& outer, size_t blocks) override;
  std::vector<F> project(const std::vector<F>& outer) override;
  void apply_images(const std::vector<F>& images) override;
  Digest fold_and_commit(const std::vector<F>& fold_weights) override;
  void sumcheck_message(F m[2]) override;
  void sumcheck_fold(F ch) override;
  F sumcheck_final_value() override;
  F sumcheck_final_weight() override;
  std::vector<uint8_t> binding_rows(const RowSelection& sel, const std::vector<Digest>& roots) override;
  const CodewordView<F>& folded_codeword() override { return *folded_; }
  const CodewordView<F>& codeword() override { return *blocks_.at(0); }
  std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    return open_top(*folded_, point, col_log);
  }
  std::vector<F> opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    return open_top(*blocks_.at(0), point, col_log);
  }
  TopRoundAccel<F>* top_round_accel() override { return this; }
  DecideAccel<F>* decide_accel() override { return this; }
  // Top opening round with the message-length vectors in HBM.
  RoundOutput<F> prove_top_round(const PcsParams<F>& pp, size_t level, const std::vector<F>& point,
                                 const std::vector<F>& opening, PcsTranscript<F>& t) override;
  bool open_round(const CodewordView<F>& cw, size_t n_rows, const std::vector<F>& point, size_t col_log,
                  std::vector<F>& opening) override {
    const auto* dc = dynamic_cast<const DeviceCodeword*>(&cw);
    if (!dc || n_rows < 1024) return false;
    opening = open_top(*dc, point, col_log);
    return true;
  }
  // Decide MultiEval (alpha columns, plus the carried message) with the row
  // vectors in HBM; declines below 1024 rows.
  bool multi_eval(const PcsParams<F>& pp, size_t level, const std::vector<EvalClaim<F>>& claims,
                  const std::vector<F>* carry_message, size_t log_rows, size_t log_cols, size_t row_factor,
                  PcsTranscript<F>& t, MultiEvalOut<F>& out) override;
  bool direct_switch(const QaCode<F>& target, size_t target_level, size_t row_factor, const RowSelection& sel,
                     const std::vector<F>& iota, const std::vector<F>& folded_message, F merged_value,
                     const std::vector<F>& merged_left, PcsTranscript<F>& t, SwitchCarry<F>& out) override;

  // EO
  void cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) override;
  F eo_build(const Query<F>& q, F challenge, F inverse, size_t logical, size_t stride) override;
  std::array<F, 2> eo_round_cross() override { return cross_; }
  void eo_round_fold(F inv, F ch) override;
  std::array<F, 2> eo_terminal() override;

  // Lane projections of arbitrary tensor terms (TBV claims and EO cross terms).
  std::vector<std::vector<F>> project_terms(const std::vector<const Term<F>*>& terms, size_t stride);
  // Raw window values of small terms.
  std::vector<int8_t> windows(const std::vector<uint64_t>& starts, size_t stride);


 private:
  // Encode the message halves of `out` with alpha (parity = WHT(alpha * WHT(msg)))
  // and build its row tree with the base- or extension-row leaf domain.
  void encode_and_hash(DeviceCodeword& out, const Fe* alpha, int logR, int logm, bool ext_domain);
  std::vector<F> open_top(const DeviceCodeword& cw, const std::vector<F>& point, size_t col_log);
  void tensor_table(const std::vector<F>& point, DBuf<Fe>& out);
  void wht_dev(Fe* v, int logn, const Fe* alpha);
  F dot_dev(const Fe* a, const Fe* b, uint64_t n);
  std::array<F, 2> lb_cross(const Fe* L, const Fe* R, uint64_t n);
  // LiteBullet (or MultiEval row rounds) on device vectors, folded in place.
  LiteBullet<F> litebullet_dev(F claimed, Fe* L, Fe* R, uint64_t n, PcsTranscript<F>& t, const char* label,
                               const char* fold_label, bool check_and_absorb);
  const Fe* level_alpha(size_t level, int which);
  void mobius_rest(Fe* cw, int logm, int logR, int from);
  std::vector<F> reduce_to_host(const DBuf<Fe>& partials, uint32_t count, int n);

  const Parameters<F>& P_;
  const int8_t* bva_;
  size_t active_;
  cudaStream_t s_;
  std::vector<std::unique_ptr<DeviceCodeword>> blocks_;
  std::vector<Digest> roots_;
  std::unique_ptr<DeviceCodeword> folded_;
  DeviceTables own_tables_;
  DeviceTables* tables_;
  const DeviceCodeword* open_cw_ = nullptr;  // codeword whose top round is being opened
  DBuf<Fe> rw_d_;                            // its row weights
  F lb_rhs_;                                 // running claim after the last device LiteBullet
  // opening state
  DBuf<Fe> weights_, values_, tmp_v_, tmp_w_;
  uint64_t sum_len_ = 0;
  bool msg_valid_ = false;
  F msg_[2];
  // EO state
  DBuf<Fe> wit_, qv_, wit2_, qv2_;
  uint64_t eo_len_ = 0;
  std::array<F, 2> cross_;
  DBuf<Fe> partials_, result_;
};

}  // namespace qfg
