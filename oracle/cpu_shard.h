// ORACLE (test infrastructure only).  One rank's part of a block-sharded
// proof, computed on the CPU by the restatement in cpu_backend.h.  It stands
// in for a rank's device in the multi-rank CPU tests of the sharding layer
// (csrc/host/sharded.h): the rank keeps a copy of the BVA in which every
// entry outside the blocks it holds is zero, so each weight-linear sum it
// returns is the part of the sum that its own blocks contribute.
#pragma once
#include "cpu_backend.h"
#include "../parcomm_b200/csrc/host/sharded.h"

namespace qf_oracle {

template <class F, class T>
struct CpuShard : ShardBackend<F> {
  const Parameters<F>& P;
  size_t lo, hi;          // held blocks [lo, hi)
  std::vector<T> masked;  // the BVA with the entries outside the held blocks zeroed
  CpuBackend<F, T> be;

  CpuShard(const Parameters<F>& p, const T* values, size_t n, const BlockShards& shards, int rank)
      : P(p), lo(shards.first(rank)), hi(shards.first(rank + 1)), masked(mask(p, values, n, lo, hi)),
        be(p, masked.data(), n) {}
  static std::vector<T> mask(const Parameters<F>& p, const T* v, size_t n, size_t lo, size_t hi) {
    std::vector<T> m(n, T(0));
    const size_t a = std::min(n, lo * p.block_len), b = std::min(n, hi * p.block_len);
    std::copy(v + a, v + b, m.begin() + a);
    return m;
  }
  void held(size_t b) const { check(b >= lo && b < hi, "block not held by this rank"); }

  Digest commit_block(size_t b) override { held(b); return be.commit_block(b); }
  std::vector<std::vector<F>> project_blocks(const std::vector<F>& outer, size_t blocks) override {
    return be.project_blocks(outer, blocks);
  }
  void apply_images(const std::vector<F>& images) override { be.apply_images(images); }
  // The block fold of packed_batch.rs:213-236 over the held blocks.
  std::vector<F> fold_part(const std::vector<F>& fw) override {
    std::vector<F> part(be.m(), F::zero());
#pragma omp parallel for if (be.m() >= 4096)
    for (long i = 0; i < long(be.m()); ++i) {
      F s = F::zero();
      for (size_t b = lo; b < hi; ++b) s += be.packed(b, i) * fw[b];
      part[i] = s;
    }
    return part;
  }
  // The folded commit of CpuBackend::fold_and_commit on the summed values.
  Digest commit_folded(std::vector<F> values) override {
    check(values.size() == be.m(), "folded values length");
    be.sum_values = values;
    mobius(values);
    be.folded = std::make_unique<Codeword<F>>(
        encode_and_commit(P.pcs.pp->seq.top(), values, P.pcs.pp->extension_columns, kLeafBaseDomain));
    return be.folded->root();
  }
  void sumcheck_message(F m[2]) override { be.sumcheck_message(m); }
  void sumcheck_fold(F ch) override { be.sumcheck_fold(ch); }
  F sumcheck_final_value() override { return be.sumcheck_final_value(); }
  F sumcheck_final_weight() override { return be.sumcheck_final_weight(); }
  void write_block_rows(ByteWriter& w, size_t b, const RowSelection& sel, const Digest& root) override {
    held(b);
    if (!be.blocks[b] || be.blocks[b]->root() != root) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
    write_codeword_rows(w, *be.blocks[b], sel);
  }
  void write_folded_rows(ByteWriter& w, const RowSelection& sel) override { write_codeword_rows(w, *be.folded, sel); }
  const CodewordView<F>& folded_codeword() override { return *be.folded; }
  std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    return be.folded_opening(point, col_log, rw);
  }

  void cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) override {
    be.cross_terms(q, stride, pos, neg);
  }
  F eo_build(const Query<F>& q, F ch, F inv, size_t logical, size_t stride) override {
    return be.eo_build(q, ch, inv, logical, stride);
  }
  std::array<F, 2> eo_round_cross() override { return be.eo_round_cross(); }
  void eo_round_fold(F inv, F ch) override { be.eo_round_fold(inv, ch); }
  std::array<F, 2> eo_terminal() override { return be.eo_terminal(); }
};

}  // namespace qf_oracle
