// CUDA implementation of the packed-PCS / EO backend for F65521^8 with int8
// weights.  All bulk data (BVA, codewords, Merkle trees, EO and sumcheck
// vectors) stays in HBM; only transcript-sized values cross to the host.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "host/protocol.h"
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
    if (count) QF_CK(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void reset() { if (p) cudaFree(p); p = nullptr; n = 0; }
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

// Constant hash prefixes computed on the host.
qfd::LeafPrefix leaf_prefix(size_t n_cols);
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

class GpuBackend : public Backend<F>, public SingleBackend<F>, public EoBackend<F> {
 public:
  GpuBackend(const Parameters<F>& p, const int8_t* d_bva, size_t active, cudaStream_t s);
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
  std::vector<F> folded_row_projection(const std::vector<F>& rw) override { return folded_->project_rows(P_.pcs.pp->top_rows(), rw); }
  std::vector<F> row_projection(const std::vector<F>& rw) override { return blocks_.at(0)->project_rows(P_.pcs.pp->top_rows(), rw); }

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

  // Kernel launches performed so far (for reporting).
  uint64_t launches = 0;

 private:
  void encode_and_hash(DeviceCodeword& out);
  void mobius_rest(Fe* cw, int logm, int logR, int from);
  std::vector<F> reduce_to_host(const DBuf<Fe>& partials, uint32_t count, int n);
  void ensure_alpha();

  const Parameters<F>& P_;
  const int8_t* bva_;
  size_t active_;
  cudaStream_t s_;
  std::vector<std::unique_ptr<DeviceCodeword>> blocks_;
  std::vector<Digest> roots_;
  std::unique_ptr<DeviceCodeword> folded_;
  DBuf<Fe> alpha1_;
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
