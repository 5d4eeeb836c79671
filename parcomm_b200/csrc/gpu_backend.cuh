// CUDA implementation of the packed-PCS / EO backend for one field: F65521^8
// with int8 weights, or KoalaBear^4 with int16 payloads when QF_FIELD_KB is
// defined (the translation unit that includes this header picks one).  All bulk
// data (BVA, codewords, Merkle trees, EO and sumcheck vectors) stays in HBM;
// only transcript-sized values cross to the host.
#pragma once
#include <functional>

#include "device/field_dev.cuh"
#include "field_select.h"
#include "gpu_common.cuh"

namespace QFD_NS {
struct TermTiles;  // kernels/open.cuh
}

namespace QFB_NS {
using namespace qf;
using namespace qfg;
namespace qfd = ::QFD_NS;
using qfd::Fe;

inline const Fe* as_fe(const F* p) { return reinterpret_cast<const Fe*>(p); }
inline Fe to_fe(const F& v) { Fe e; std::memcpy(&e, &v, 16); return e; }
inline F from_fe(const Fe& e) { F v; std::memcpy(&v, &e, 16); return v; }

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

// Weights held in host memory (the caller's buffer; pinned memory lets the
// copies run at full speed and ahead of the compute) and staged into HBM one
// PCS block at a time for every pass that reads them: the reference's
// recompute mode, for weight sets larger than HBM.  The first `resident`
// blocks are copied on the first pass and stay in HBM; the others cycle
// through `slots` staging buffers, copied on a side stream while earlier
// blocks are processed.
class BlockStream {
 public:
  BlockStream(const W* host, uint64_t active, uint64_t block_len, size_t resident, int slots);
  ~BlockStream();
  BlockStream(const BlockStream&) = delete;
  BlockStream& operator=(const BlockStream&) = delete;
  uint64_t active() const { return active_; }
  uint64_t block_len() const { return block_len_; }
  // The weights are already in HBM (a device pointer): every block is used in
  // place and nothing is copied.
  bool on_device() const { return device_; }
  size_t live_blocks() const { return live_; }
  size_t resident_blocks() const { return resident_; }
  const W* host() const { return host_; }  // the weights (device memory when on_device())
  uint64_t h2d_bytes() const { return copied_; }
  // fn(b, d, n) for every live block b, with its launches on `s`: d is the
  // device copy of entries [b * block_len, b * block_len + n).  After the
  // first (ascending) pass, a pass starts with the blocks the previous pass
  // left staged and interleaves the other streamed blocks with the resident
  // ones; callers must not depend on the order.  Weights already in HBM are
  // visited in ascending order.
  using BlockFn = std::function<void(size_t b, const W* d, uint64_t n)>;
  void for_each(cudaStream_t s, const BlockFn& fn);

 private:
  const W* host_;
  uint64_t active_, block_len_;
  size_t live_, resident_;
  bool device_ = false;
  bool resident_ready_ = false;
  DBuf<W> resident_buf_;
  std::vector<DBuf<W>> slot_buf_;
  std::vector<cudaEvent_t> landed_;  // per live block: its copy has landed
  std::vector<cudaEvent_t> freed_;   // per slot: the compute on its last block is done
  std::vector<size_t> slot_block_;   // per slot: the block its last copy staged
  cudaStream_t copy_ = nullptr;
  uint64_t copied_ = 0;
};

// Commitment root of block `b` of a device BVA (`active` entries), computed
// only in the caller's device buffers: `cw` holds 2R x cols entries, `tree`
// 4 x 2R words (2 x 2R digests), `alpha` the R entries of the top code's
// alpha table (alphas[1]), already on the device.  Launches on `s`, writes the
// 32-byte root to the device bytes `d_root` and returns without
// synchronising; allocates no device memory.
void commit_block_into(const Parameters<F>& P, const W* d_bva, uint64_t active, size_t b, Fe* cw, uint4* tree,
                       const Fe* alpha, uint8_t* d_root, cudaStream_t s);

// The setup commitments of a parameter set on the current device
// (ShortQaFoldPC::setup, qafold_short_pc.rs:401-444; direct-interleaved
// setup, qafold_short_setup.rs:427-536): each level's columns are encoded by
// the commit's transform passes and its rows hashed by k_hash_setup_rows;
// the host keeps the encoded matrix and builds the tree from the leaves.
// Levels below 2^20 encoded entries stay on the host.
class DeviceSetup final : public SetupAccel<F> {
 public:
  bool encode_level(const QaCode<F>& target, const QaCode<F>& current, size_t row_factor, const SetupShape& shape,
                    std::vector<F>& encoded, std::vector<Digest>& leaves) override;
};

class GpuBackend : public Backend<F>,
                   public SingleBackend<F>,
                   public EoBackend<F>,
                   public TopRoundAccel<F>,
                   public DecideAccel<F> {
 public:
  // `tables` (optional, not owned) shares uploaded code tables across backends.
  GpuBackend(const Parameters<F>& p, const W* d_bva, size_t active, cudaStream_t s, DeviceTables* tables = nullptr);
  // Streamed weights (not owned): only block roots stay in HBM, and binding
  // re-encodes every block.
  GpuBackend(const Parameters<F>& p, BlockStream* src, cudaStream_t s, DeviceTables* tables = nullptr);
  // Commits every block of a streamed backend in one pass over the weights;
  // `per_block` runs after each live block's launches (same stream).
  std::vector<Digest> commit_streamed(const BlockStream::BlockFn& per_block);
  // Returns the buffers of the last opening (tables, folded codeword, the
  // sumcheck and EO vectors, a re-encoded block) to the pool: a commitment
  // that waits for its next opening keeps only its own weights, codewords
  // and trees.
  void release_opening_state();
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
  const CodewordView<F>& codeword() override { return single_codeword(); }
  std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    return open_top(*folded_, point, col_log);
  }
  std::vector<F> opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    return open_top(single_codeword(), point, col_log);
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
  // Decide carry commitment on the device for codes of at least 128 rows.
  std::unique_ptr<CodewordView<F>> commit_carry(const PcsParams<F>& pp, size_t code_index, const std::vector<F>& message,
                                                size_t n_cols) override;

  // EO
  void cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) override;
  F eo_build(const Query<F>& q, F challenge, F inverse, size_t logical, size_t stride) override;
  std::array<F, 2> eo_round_cross() override { return cross_; }
  void eo_round_fold(F inv, F ch) override;
  std::array<F, 2> eo_terminal() override;

  // Lane projections of arbitrary tensor terms (TBV claims and EO cross terms).
  std::vector<std::vector<F>> project_terms(const std::vector<const Term<F>*>& terms, size_t stride);
  // The same for several groups of terms (each group with one lane width), in
  // one pass over streamed weights.
  std::vector<std::vector<std::vector<F>>> project_term_groups(const std::vector<std::vector<const Term<F>*>>& groups,
                                                               size_t stride);
  // Raw window values of small terms.
  std::vector<W> windows(const std::vector<uint64_t>& starts, size_t stride);
  // Block-sharded proofs (host/sharded.h).  The backend then holds a copy of
  // the BVA in which the blocks its rank does not hold are zero.
  // This rank's part of sum_b fold[b] * packed(b, .), on the host.
  std::vector<F> fold_values(const std::vector<F>& fold_weights);
  // The folded values summed over the ranks: kept for the sumcheck, Mobius
  // transformed, encoded and hashed as fold_and_commit does; returns the root.
  Digest commit_folded_values(const std::vector<F>& values);
  // The binding rows of committed block b (whose root must be `root`) and of
  // the folded codeword, in the batch payload's format.
  void write_block_rows(ByteWriter& w, size_t b, const RowSelection& sel, const Digest& root);
  void write_folded_rows(ByteWriter& w, const RowSelection& sel);

  // LogUp range audit (not part of the proof): sum_i 1 / (alpha - v_i) over
  // the weights as {numerator, denominator}, and `mult` = the multiplicity of
  // each table value (bin k: the value k - 128 for int8, k - 32768 for int16).
  std::array<F, 2> range_audit(const F& alpha, std::vector<uint64_t>& mult);


 private:
  // Encode the message halves of `out` with alpha (parity = WHT(alpha * WHT(msg)))
  // and build its row tree with the base- or extension-row leaf domain.  When
  // mob_from >= 0 the message holds the packed message with only its Mobius
  // levels [0, mob_from) applied, and the encode finishes the transform.
  void encode_and_hash(DeviceCodeword& out, const Fe* alpha, int logR, int logm, bool ext_domain, int mob_from = -1);
  std::vector<F> open_top(const DeviceCodeword& cw, const std::vector<F>& point, size_t col_log);
  void tensor_table(const std::vector<F>& point, DBuf<Fe>& out);
  void wht_dev(Fe* v, int logn, const Fe* alpha);
  F dot_dev(const Fe* a, const Fe* b, uint64_t n);
  std::array<F, 2> lb_cross(const Fe* L, const Fe* R, uint64_t n);
  // LiteBullet (or MultiEval row rounds) on device vectors, folded in place
  // down to 512 elements and on the host from there (L and R are left
  // partly folded).
  LiteBullet<F> litebullet_dev(F claimed, Fe* L, Fe* R, uint64_t n, PcsTranscript<F>& t, const char* label,
                               const char* fold_label, bool check_and_absorb);
  const Fe* level_alpha(size_t level, int which);
  // Pack + Mobius + encode + hash of the block whose entries [src_base,
  // src_base + 2^chunk) are read from `bva` (zero at or past `active`).
  Digest encode_block(const W* bva, uint64_t active, uint64_t src_base, DeviceCodeword& cw);
  DeviceCodeword& scratch_codeword();
  // Weights that reach HBM block by block (host memory); resident weights,
  // streamed or not, take the whole-array launches.
  bool streaming() const { return src_ && !src_->on_device(); }
  // The codeword of a single-block statement (re-encoded once per opening
  // for streamed weights).
  const DeviceCodeword& single_codeword();
  std::vector<std::vector<std::vector<F>>> project_groups_streamed(const std::vector<std::vector<const Term<F>*>>& groups,
                                                                   size_t stride);
  std::vector<F> reduce_to_host(const DBuf<Fe>& partials, uint32_t count, int n);
  std::vector<F> copy_to_host(const Fe* p, uint64_t n);
  void block_fold_launch(const W* bva, uint64_t active, int blocks, const Fe* T, int accumulate);
  void project_terms_launch(const W* bva, uint64_t active, const qfd::TermTiles* terms, int n_terms, uint64_t tiles,
                            const Fe* tables, size_t lanes, Fe* out, uint64_t bytes);
  void eq_project_launch(const W* bva, uint64_t active, uint64_t b0, int nb, unsigned long long* raw, unsigned grid);
  void eo_witness_launch(const W* bva, uint64_t active, uint64_t rows, size_t stride, const Fe* powers, Fe* out);

  const Parameters<F>& P_;
  const W* bva_;              // resident weights, or null
  BlockStream* src_ = nullptr;  // streamed weights, or null
  std::unique_ptr<DeviceCodeword> scratch_;  // re-encoded block of a streamed backend
  const DeviceCodeword* single_cw_ = nullptr;  // this opening's re-encoded single block
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
  std::vector<F> host_v_, host_w_;  // the sumcheck's last rounds (length <= kHostTail), on the host
  // EO state
  DBuf<Fe> wit_, qv_, wit2_, qv2_;
  uint64_t eo_len_ = 0;
  std::array<F, 2> cross_;
  std::vector<F> host_wit_, host_qv_;  // the EO's last binary rounds, on the host
  DBuf<Fe> partials_;  // reduction buffer: header (counter, result) + one slot per CTA
};

}  // namespace QFB_NS
