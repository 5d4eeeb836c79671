// ORACLE (test infrastructure only).  A plain CPU restatement of every
// data-parallel step that the CUDA library computes: weight packing, the
// Mobius transform, QA encoding + Merkle commitment, TBV lane projections and
// Laurent cross terms, the packed EO witness / query fold / binary rounds,
// the equality-table lane projection, weight images, block fold, degree-2
// sumcheck and the codeword-fold binding payload.
//
// Each function follows the reference loop it names; exact field arithmetic
// makes evaluation order irrelevant.  Only tests, `__graft_entry__.smoke()`
// and the bench's CPU-baseline leg may load this code, to compare results with.
#pragma once
#include <memory>
#include <vector>

#include "../parcomm_b200/csrc/host/protocol.h"

namespace qf_oracle {
using namespace qf;

// mobius_in_place (packed.rs:708-752): high[i] -= low[i] at every level.
template <class F>
void mobius(std::vector<F>& v) {
  size_t n = v.size();
  // Butterfly k of a level pairs i = (k / half) * 2 half + k % half with
  // i + half, so every level spreads over the threads (the top levels too).
  for (size_t half = 1, lh = 0; half < n; half <<= 1, ++lh)
#pragma omp parallel for schedule(static) if (n >= (1u << 16))
    for (long k = 0; k < long(n / 2); ++k) {
      const size_t i = ((size_t(k) >> lh) << (lh + 1)) | (size_t(k) & (half - 1));
      v[i + half] -= v[i];
    }
}

template <class F, class T>
struct CpuBackend : Backend<F>, SingleBackend<F>, EoBackend<F> {
  const Parameters<F>& P;
  const T* values;  // BVA, `active` entries, implicit zero suffix
  size_t active;
  std::vector<std::unique_ptr<Codeword<F>>> blocks;  // committed block codewords
  std::vector<F> weights, sum_values;
  std::unique_ptr<Codeword<F>> folded;
  std::vector<F> witness, query_values;

  CpuBackend(const Parameters<F>& p, const T* v, size_t n) : P(p), values(v), active(n) {}

  uint32_t small_at(size_t g) const { return g < active ? F::small(int(values[g])) : 0u; }
  F packed(size_t block, size_t i) const {
    F r;
    const size_t base = block * P.block_len + i * F::kLanes;
    for (int l = 0; l < F::kLanes; ++l) r.c[l] = typename F::Coeff(small_at(base + l));
    return r;
  }
  size_t m() const { return P.pcs.packed_len(); }

  // ---- commit: pack -> Mobius -> QA encode -> row hashes -> tree
  Digest commit_block(size_t b) override {
    std::vector<F> coeff(m());
#pragma omp parallel for if (m() >= 4096)
    for (long i = 0; i < long(m()); ++i) coeff[i] = packed(b, i);
    mobius(coeff);
    if (blocks.size() <= b) blocks.resize(b + 1);
    blocks[b] = std::make_unique<Codeword<F>>(
        encode_and_commit(P.pcs.pp->seq.top(), coeff, P.pcs.pp->extension_columns, kLeafBaseDomain));
    return blocks[b]->root();
  }
  Digest commit() override { return commit_block(0); }

  // ---- equality-table lane projection (project_lanes_from_fn, packed_batch.rs:25-41)
  std::vector<F> lanes_of(size_t b) const {
    std::vector<F> lanes(F::kLanes, F::zero());
#pragma omp parallel
    {
      std::vector<F> local(F::kLanes, F::zero());
#pragma omp for nowait
      for (long i = 0; i < long(m()); ++i) {
        const F v = packed(b, i);
        for (int j = 0; j < F::kLanes; ++j) local[j] += weights[i].mul_prime(v.c[j]);
      }
#pragma omp critical
      for (int j = 0; j < F::kLanes; ++j) lanes[j] += local[j];
    }
    return lanes;
  }
  std::vector<std::vector<F>> project_blocks(const std::vector<F>& outer, size_t nblocks) override {
    weights = equality_table(outer);
    std::vector<std::vector<F>> out;
    for (size_t b = 0; b < nblocks; ++b) out.push_back(lanes_of(b));
    return out;
  }
  std::vector<F> project(const std::vector<F>& outer) override {
    weights = equality_table(outer);
    sum_values.resize(m());
    for (size_t i = 0; i < m(); ++i) sum_values[i] = packed(0, i);
    return lanes_of(0);
  }
  // apply_weight_images (packed.rs:634-650): w <- sum_j w.c[j] * images[j]
  void apply_images(const std::vector<F>& images) override {
#pragma omp parallel for if (weights.size() >= 4096)
    for (long i = 0; i < long(weights.size()); ++i) {
      F s = F::zero();
      for (int j = 0; j < F::kLanes; ++j) s += images[j].mul_prime(weights[i].c[j]);
      weights[i] = s;
    }
  }
  // block fold + folded commit (packed_batch.rs:213-236)
  Digest fold_and_commit(const std::vector<F>& fw) override {
    sum_values.assign(m(), F::zero());
#pragma omp parallel for if (m() >= 4096)
    for (long i = 0; i < long(m()); ++i) {
      F s = F::zero();
      for (size_t b = 0; b < fw.size(); ++b) s += packed(b, i) * fw[b];
      sum_values[i] = s;
    }
    std::vector<F> coeff = sum_values;
    mobius(coeff);
    folded = std::make_unique<Codeword<F>>(
        encode_and_commit(P.pcs.pp->seq.top(), coeff, P.pcs.pp->extension_columns, kLeafBaseDomain));
    return folded->root();
  }
  // round_message / fold_pair (packed.rs:652-696)
  void sumcheck_message(F msg[2]) override {
    const long h = long(sum_values.size() / 2);
    F a = F::zero(), b = F::zero();
#pragma omp parallel if (h >= 4096)
    {
      F la = F::zero(), lb = F::zero();
#pragma omp for nowait
      for (long i = 0; i < h; ++i) {
        la += sum_values[i] * weights[i];
        lb += (sum_values[i + h] - sum_values[i]) * (weights[i + h] - weights[i]);
      }
#pragma omp critical
      {
        a += la;
        b += lb;
      }
    }
    msg[0] = a;
    msg[1] = b;
  }
  void sumcheck_fold(F ch) override {
    const long h = long(sum_values.size() / 2);
    // Index i reads i and i + h and writes i < h: disjoint per i.
#pragma omp parallel for if (h >= 4096)
    for (long i = 0; i < h; ++i) {
      sum_values[i] = sum_values[i] + ch * (sum_values[i + h] - sum_values[i]);
      weights[i] = weights[i] + ch * (weights[i + h] - weights[i]);
    }
    sum_values.resize(h);
    weights.resize(h);
  }
  F sumcheck_final_value() override { return sum_values[0]; }
  F sumcheck_final_weight() override { return weights[0]; }
  // prove_codeword_fold(_recomputed) payload (qafold_short_batch.rs:77-160)
  std::vector<uint8_t> binding_rows(const RowSelection& sel, const std::vector<Digest>& roots) override {
    ByteWriter w;
    w.bytes("QAFOLDB1", 8);
    w.len(roots.size());
    for (size_t b = 0; b < roots.size(); ++b) {
      if (blocks[b]->root() != roots[b]) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
      write_codeword_rows(w, *blocks[b], sel);
    }
    write_codeword_rows(w, *folded, sel);
    return std::move(w.out);
  }
  const CodewordView<F>& folded_codeword() override { return *folded; }
  const CodewordView<F>& codeword() override { return *blocks[0]; }
  std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    rw = tensor_weights(std::vector<F>(point.begin() + col_log, point.end()));
    return systematic_row_projection(*folded, P.pcs.pp->top_rows(), rw);
  }
  std::vector<F> opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    rw = tensor_weights(std::vector<F>(point.begin() + col_log, point.end()));
    return systematic_row_projection(*blocks[0], P.pcs.pp->top_rows(), rw);
  }

  // ---- EO (tbv.rs:288-428, eo.rs:97-181)
  std::vector<F> project_term(const Term<F>& term, size_t stride) const {
    size_t low_bits = std::min<size_t>(ilog2(stride), term.factors.size());
    size_t lanes = size_t(1) << low_bits;
    std::vector<F> out(lanes, F::zero());
    if (term.offset >= active || term.scale.is_zero()) return out;
    std::vector<F> hw = factor_weights(term.factors.data() + low_bits, term.factors.size() - low_bits);
    size_t rows = std::min((active - term.offset + lanes - 1) / lanes, term.len() / lanes);
    std::vector<F> sums(lanes, F::zero());
#pragma omp parallel if (rows * lanes >= 4096)
    {
      std::vector<F> local(lanes, F::zero());
#pragma omp for nowait
      for (long r = 0; r < long(rows); ++r)
        for (size_t lane = 0; lane < lanes; ++lane) {
          size_t idx = term.offset + r * lanes + lane;
          if (idx < active && values[idx] != 0) local[lane] += hw[r].mul_prime(F::small(int(values[idx])));
        }
#pragma omp critical
      for (size_t lane = 0; lane < lanes; ++lane) sums[lane] += local[lane];
    }
    for (size_t lane = 0; lane < lanes; ++lane) out[lane] = sums[lane] * term.scale;
    return out;
  }
  void cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) override {
    pos.assign(stride - 1, F::zero());
    neg.assign(stride - 1, F::zero());
    for (const Term<F>& term : q.terms) {
      if (term.len() >= stride) {
        std::vector<F> pr = project_term(term, stride);
        std::vector<F> low = factor_weights(term.factors.data(), ilog2(stride));
        for (size_t d = 1; d < stride; ++d)
          for (size_t lane = 0; lane + d < stride; ++lane) {
            pos[d - 1] += pr[lane] * low[lane + d];
            neg[d - 1] += pr[lane + d] * low[lane];
          }
      } else {
        size_t start = term.offset / stride * stride;
        std::vector<F> qv(stride, F::zero());
        for (size_t i = 0; i < term.len(); ++i) qv[term.offset - start + i] = term.weight(i);
        for (size_t d = 1; d < stride; ++d)
          for (size_t lane = 0; lane + d < stride; ++lane) {
            pos[d - 1] += qv[lane + d].mul_prime(small_at(start + lane));
            neg[d - 1] += qv[lane].mul_prime(small_at(start + lane + d));
          }
      }
    }
  }
  F eo_build(const Query<F>& q, F ch, F inv, size_t logical, size_t stride) override {
    std::vector<F> powers_inv = consecutive_powers(inv, stride);
    witness.assign(logical / stride, F::zero());
#pragma omp parallel for if (logical >= (1u << 16))
    for (long row = 0; row < long(logical / stride); ++row) {
      F s = F::zero();
      for (size_t lane = 0; lane < stride; ++lane) {
        uint32_t v = small_at(row * stride + lane);
        if (v) s += powers_inv[lane].mul_prime(v);
      }
      witness[row] = s;
    }
    // Query::fold (tbv.rs:393-428)
    query_values.assign(logical / stride, F::zero());
    std::vector<F> powers = consecutive_powers(ch, stride);
    for (const Term<F>& term : q.terms) {
      if (term.len() >= stride) {
        size_t lb = ilog2(stride);
        std::vector<F> low = factor_weights(term.factors.data(), lb);
        F sc = F::zero();
        for (size_t j = 0; j < stride; ++j) sc += low[j] * powers[j];
        sc = term.scale * sc;
        std::vector<F> hw = factor_weights(term.factors.data() + lb, term.factors.size() - lb);
        const size_t start = term.offset / stride;
#pragma omp parallel for if (hw.size() >= 4096)
        for (long i = 0; i < long(hw.size()); ++i) query_values[start + i] += sc * hw[i];
      } else {
        for (size_t i = 0; i < term.len(); ++i) query_values[term.offset / stride] += term.weight(i) * powers[(term.offset + i) % stride];
      }
    }
    F dot = F::zero();
    const long nw = long(witness.size());
#pragma omp parallel if (nw >= 4096)
    {
      F local = F::zero();
#pragma omp for nowait
      for (long i = 0; i < nw; ++i) local += witness[i] * query_values[i];
#pragma omp critical
      dot += local;
    }
    return dot;
  }
  std::array<F, 2> eo_round_cross() override {
    F a = F::zero(), b = F::zero();
    const long pairs = long(witness.size() / 2);
#pragma omp parallel if (pairs >= 4096)
    {
      F la = F::zero(), lb = F::zero();
#pragma omp for nowait
      for (long j = 0; j < pairs; ++j) {
        la += witness[2 * j] * query_values[2 * j + 1];
        lb += witness[2 * j + 1] * query_values[2 * j];
      }
#pragma omp critical
      {
        a += la;
        b += lb;
      }
    }
    return {a, b};
  }
  void eo_round_fold(F inv, F ch) override {
    const long h = long(witness.size() / 2);
    // Out of place: index i reads 2i and 2i + 1.
    std::vector<F> w(h), q(h);
#pragma omp parallel for if (h >= 4096)
    for (long i = 0; i < h; ++i) {
      w[i] = witness[2 * i] + witness[2 * i + 1] * inv;
      q[i] = query_values[2 * i] + query_values[2 * i + 1] * ch;
    }
    witness.swap(w);
    query_values.swap(q);
  }
  std::array<F, 2> eo_terminal() override { return {witness[0], query_values[0]}; }
};

// tbv::evaluate_claims (tbv.rs:143-185) over the BVA.
template <class F, class T>
std::vector<Claim<F>> evaluate_claims(const Parameters<F>& P, const T* values, size_t n,
                                      const std::vector<std::pair<std::vector<F>, std::vector<F>>>& points) {
  check(n == P.layout.active && points.size() == P.layout.shapes.size(), "claim input dimensions");
  std::vector<Claim<F>> claims;
  for (const auto& p : points) claims.push_back({p.first, p.second, F::zero()});
  validate_claims(P.layout, claims);
  CpuBackend<F, T> be(P, values, n);
  for (const Bucket& b : P.layout.buckets) {
    const auto& row = points[b.matrix].first;
    const auto& col = points[b.matrix].second;
    Term<F> term{b.offset, monomial_weight(b.row_offset, row.data(), row.size()) * monomial_weight(b.col_offset, col.data(), col.size()), {}};
    for (int k = 0; k < ilog2(b.cols); ++k) term.factors.push_back({F::one(), col[k]});
    for (int k = 0; k < ilog2(b.rows); ++k) term.factors.push_back({F::one(), row[k]});
    std::vector<F> partial = be.project_term(term, 16);
    std::vector<F> low = factor_weights(term.factors.data(), std::min<size_t>(4, term.factors.size()));
    F v = F::zero();
    for (size_t i = 0; i < partial.size(); ++i) v += partial[i] * low[i];
    claims[b.matrix].value += v;
  }
  return claims;
}

// Full prover: commit every block, then prove (protocol.rs:131-263).
template <class F, class T>
struct ProveResult {
  Commitment statement;
  std::vector<Claim<F>> claims;
  Proof<F> proof;
  std::vector<uint8_t> wire;
  StageTimes times;
  double commit_ms = 0, open_ms = 0;
};

template <class F, class T>
ProveResult<F, T> prove_all(const Parameters<F>& P, const T* values, size_t n, bool benchmark_claims,
                            const std::vector<Claim<F>>* given_claims = nullptr) {
  validate_values(P.layout, values, n);
  CpuBackend<F, T> be(P, values, n);
  ProveResult<F, T> out;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<Digest> roots;
  for (size_t b = 0; b < P.blocks(); ++b) roots.push_back(be.commit_block(b));
  out.commit_ms = ms_since(t0);
  out.statement = make_statement(P, roots);
  if (benchmark_claims) out.claims = evaluate_claims(P, values, n, benchmark_points<F>(out.statement));
  else out.claims = *given_claims;
  t0 = std::chrono::steady_clock::now();
  Transcript<F> t = statement_transcript(P, out.statement, out.claims);
  Query<F> q = compile(P.layout, out.claims, t);
  auto [eo, term] = eo_prove<F>(be, P.layout.logical, size_t(1) << P.config.packed_log, q, t);
  std::vector<uint8_t> ctx = opening_context<F>(t.state, 0);
  BatchOpening<F> op = roots.size() > 1 ? open_batch(P.pcs, be, roots, term.point_msb, ctx)
                                        : open_single(P.pcs, be, roots[0], term.point_msb, ctx);
  check(op.claimed_value * term.scale == term.value, "QAFold/EO terminal mismatch");
  out.proof.eo = eo;
  out.proof.opening_value = op.claimed_value;
  out.proof.opening_proof = std::move(op.wire);
  out.wire = proof_to_bytes(out.proof);
  out.open_ms = ms_since(t0);
  out.times = op.times;
  return out;
}

}  // namespace qf_oracle
