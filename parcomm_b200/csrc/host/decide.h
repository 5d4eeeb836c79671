// Recursive Decide for the direct-interleaved setup: authenticates every
// deferred generator claim of a QAFold opening against the setup commitments.
//
// Reference: driver (qafold_short_decide_driver.rs:28-797), claim preparation
// (qafold_short_decide_protocol.rs:92-387), MultiEval
// (qafold_short_decide.rs:53-560), direct-interleaved carries, iota and code
// switch (qafold_short_decide_carry.rs:118-262, 329-760, 940-1352), the
// G-to-H reduction (qafold_short.rs:1538-1604) and the wire
// (qafold_short_decide_wire.rs).  Only DirectInterleavedV1 is reachable for
// the supported fields, so the RF-code branches are not restated.
#pragma once
#include <exception>
#include <mutex>
#include <optional>
#include <vector>

#include "pcs.h"

namespace qf {

template <class F>
struct MatrixClaim {
  F value;
  std::vector<F> left, right;  // point.0, point.1
};
template <class F>
struct EvalClaim {
  F value;
  std::vector<F> row_point;
  std::vector<F> col_weight;
};
template <class F>
struct EvalWithPoint {
  F value;
  std::vector<F> point;
};

// reduce_short_generator_claim: G_j claim -> H_j (alpha matrix) claim.
template <class F>
MatrixClaim<F> reduce_generator_claim(size_t message_len, size_t index, const MatrixClaim<F>& c) {
  size_t lm = ilog2(message_len), li = ilog2(index);
  if (c.left.size() != lm + li || c.right.size() != lm) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "generator claim dims");
  std::vector<F> block_point(c.left.begin(), c.left.begin() + li);
  std::vector<F> left_msg(c.left.begin() + li, c.left.end());
  auto transform = [](const std::vector<F>& p, F& norm, std::vector<F>& out) {
    norm = F::one();
    for (const F& v : p) {
      F d = F::one() + v;
      F inv;
      if (!d.try_inverse(inv)) fail(QF_E_INVALID_COMMITMENT, "wht point");
      norm *= d;
      out.push_back((F::one() - v) * inv);
    }
  };
  F ln, rn;
  std::vector<F> tl, tr;
  transform(left_msg, ln, tl);
  transform(c.right, rn, tr);
  F norm = ln * rn;
  F inv;
  if (!norm.try_inverse(inv)) fail(QF_E_INVALID_COMMITMENT, "normalization");
  MatrixClaim<F> out;
  out.value = c.value * inv;
  for (size_t i = 0; i < tl.size(); ++i) out.left.push_back(tl[i] * tr[i]);
  out.right = block_point;
  return out;
}

// ------------------------------------------------------------ wire structs
template <class F>
struct SetupRowQuery {
  size_t row_index;
  std::vector<F> row;
  Path path;
};
template <class F>
struct SetupRows {
  bool all = false;
  std::vector<SetupRowQuery<F>> partial;
  std::vector<F> encoded;
  SetupShape shape;
};
template <class F>
struct DecideRound {
  size_t level;
  std::optional<Digest> next_carry_root;
  SetupRows<F> setup_rows;
  std::optional<Rows<F>> carry_rows;
};
template <class F>
struct DecideProof {
  std::vector<F> responses;
  std::vector<DecideRound<F>> rounds;
  std::vector<F> base_vector;
};

inline void write_shape(ByteWriter& w, const SetupShape& s) {
  s.validate();
  for (size_t v : {s.level, s.encoded_rows, s.message_rows, s.t_cols, s.t_elements, s.t_last_len, s.h_cols}) w.len(v);
}
template <class F>
std::vector<uint8_t> decide_to_bytes(const DecideProof<F>& p) {
  ByteWriter w;
  w.bytes("QFSDCID1", 8);
  w.len(p.responses.size());
  for (const F& v : p.responses) w.field(v);
  w.len(p.rounds.size());
  for (const auto& r : p.rounds) {
    w.len(r.level);
    if (r.next_carry_root) { w.u8(1); w.digest(*r.next_carry_root); } else w.u8(0);
    if (!r.setup_rows.all) {
      w.u8(0);
      w.len(r.setup_rows.partial.size());
      for (const auto& q : r.setup_rows.partial) {
        w.len(q.row_index);
        w.len(q.row.size());
        for (const F& v : q.row) w.field(v);
        write_path<F>(w, q.path);
      }
    } else {
      w.u8(1);
      write_shape(w, r.setup_rows.shape);
      w.len(r.setup_rows.encoded.size());
      for (const F& v : r.setup_rows.encoded) w.field(v);
    }
    if (r.carry_rows) { w.u8(1); write_rows(w, *r.carry_rows); } else w.u8(0);
  }
  w.len(p.base_vector.size());
  for (const F& v : p.base_vector) w.field(v);
  return std::move(w.out);
}
template <class F>
DecideProof<F> decide_from_bytes(const uint8_t* d, size_t n) {
  ByteReader r(d, n);
  if (std::memcmp(r.take(8), "QFSDCID1", 8) != 0) fail(QF_E_INVALID_COMMITMENT, "decide magic");
  DecideProof<F> p;
  uint64_t nr = r.len();
  if (nr > r.remaining() / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "decide responses");
  for (uint64_t i = 0; i < nr; ++i) p.responses.push_back(r.field<F>());
  uint64_t rounds = r.len();
  if (rounds > (r.remaining() >= 8 ? r.remaining() - 8 : 0) / 19) fail(QF_E_INVALID_COMMITMENT, "decide rounds");
  for (uint64_t i = 0; i < rounds; ++i) {
    DecideRound<F> dr;
    dr.level = r.len();
    uint8_t opt = r.u8();
    if (opt == 1) dr.next_carry_root = r.digest();
    else if (opt != 0) fail(QF_E_INVALID_COMMITMENT, "optional root tag");
    uint8_t mode = r.u8();
    if (mode == 0) {
      uint64_t q = r.len();
      if (q > r.remaining() / 16) fail(QF_E_INVALID_COMMITMENT, "setup rows");
      for (uint64_t j = 0; j < q; ++j) {
        SetupRowQuery<F> sq;
        sq.row_index = r.len();
        uint64_t len = r.len();
        if (r.remaining() < 8 || len > (r.remaining() - 8) / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "setup row len");
        for (uint64_t k = 0; k < len; ++k) sq.row.push_back(r.field<F>());
        sq.path = read_path(r);
        if (sq.row.empty()) fail(QF_E_INVALID_COMMITMENT, "empty setup row");
        dr.setup_rows.partial.push_back(std::move(sq));
      }
    } else if (mode == 1) {
      dr.setup_rows.all = true;
      SetupShape& s = dr.setup_rows.shape;
      s.level = r.len(); s.encoded_rows = r.len(); s.message_rows = r.len(); s.t_cols = r.len();
      s.t_elements = r.len(); s.t_last_len = r.len(); s.h_cols = r.len();
      try { s.validate(); } catch (const QfError&) { fail(QF_E_INVALID_COMMITMENT, "setup shape"); }
      uint64_t len = r.len();
      if (len > r.remaining() / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "setup all rows");
      for (uint64_t k = 0; k < len; ++k) dr.setup_rows.encoded.push_back(r.field<F>());
      if (s.level != dr.level || dr.setup_rows.encoded.size() != s.encoded_rows * s.total_cols())
        fail(QF_E_INVALID_COMMITMENT, "setup all rows shape");
    } else {
      fail(QF_E_INVALID_COMMITMENT, "setup rows mode");
    }
    uint8_t copt = r.u8();
    if (copt == 1) dr.carry_rows = read_rows<F>(r);
    else if (copt != 0) fail(QF_E_INVALID_COMMITMENT, "carry tag");
    if (dr.level == 0) fail(QF_E_INVALID_COMMITMENT, "decide level");
    p.rounds.push_back(std::move(dr));
  }
  uint64_t nb = r.len();
  if (nb > r.remaining() / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "decide base");
  for (uint64_t i = 0; i < nb; ++i) p.base_vector.push_back(r.field<F>());
  if (!r.empty()) fail(QF_E_INVALID_COMMITMENT, "trailing decide bytes");
  return p;
}

// ------------------------------------------------------------ MultiEval
template <class F>
struct MultiEvalOut {
  bool ok;
  EvalWithPoint<F> reduced;
  std::vector<F> folded_vector;
};

template <class F>
void absorb_multi_eval_statement(const std::vector<EvalClaim<F>>& claims, size_t log_rows, size_t log_cols, PcsTranscript<F>& t) {
  t.absorb_str("multi-eval-domain", "qafold-short-decide/multi-eval/v2");
  t.absorb_u64("multi-eval-log-rows", log_rows);
  t.absorb_u64("multi-eval-log-cols", log_cols);
  t.absorb_u64("multi-eval-claim-count", claims.size());
  for (const auto& c : claims) {
    t.absorb_ext("multi-eval-claim-value", c.value);
    t.absorb_exts("multi-eval-row-point", c.row_point);
    t.absorb_exts("multi-eval-column-weight", c.col_weight);
  }
}

template <class F>
F expected_weight_eval(const std::vector<EvalClaim<F>>& claims, const std::vector<F>& powers, size_t log_cols,
                       const std::vector<F>& point) {
  std::vector<F> cp(point.begin(), point.begin() + log_cols), rp(point.begin() + log_cols, point.end());
  std::vector<F> ct = tensor_weights(cp);
  F sum = F::zero();
  for (size_t i = 0; i < claims.size(); ++i) {
    F ce = F::zero();
    for (size_t j = 0; j < claims[i].col_weight.size() && j < ct.size(); ++j) ce += claims[i].col_weight[j] * ct[j];
    sum += powers[i] * ce * tensor_inner_product(claims[i].row_point, rp);
  }
  return sum;
}

// Column phase of MultiEval (qafold_short_decide.rs:476-505): given the
// source evaluations se[claim][source], folds the logical columns and the
// claims' column weights, pushing the cross messages.  Afterwards the folded
// matrix column is sum(coef * source) over `terms0`, and the row weight vector
// is sum_i row_scale[i] * tensor_weights(claims[i].row_point).
template <class F>
struct MultiEvalColumns {
  F rhs;
  std::vector<F> powers, row_scale, a_point, b_point;
  std::vector<std::pair<size_t, F>> terms0;
};
template <class F>
MultiEvalColumns<F> multi_eval_columns(const std::vector<EvalClaim<F>>& claims, size_t real, size_t log_cols, F rho,
                                       const std::vector<std::vector<F>>& se, PcsTranscript<F>& t) {
  const size_t cols = size_t(1) << log_cols;
  MultiEvalColumns<F> out;
  out.rhs = F::zero();
  F power = F::one();
  for (const auto& c : claims) { out.powers.push_back(power); out.rhs += power * c.value; power *= rho; }
  // Column terms: each logical column is a linear combination of sources.
  std::vector<std::vector<std::pair<size_t, F>>> terms(real);
  for (size_t c = 0; c < real; ++c) terms[c].push_back({c, F::one()});
  std::vector<std::vector<F>> cw;  // column weight state per claim
  for (const auto& c : claims) cw.push_back(c.col_weight);
  size_t logical = cols;
  auto eval_at = [&](size_t column, size_t claim) {
    F s = F::zero();
    if (column < terms.size())
      for (const auto& [src, coef] : terms[column]) s += se[claim][src] * coef;
    return s;
  };
  auto wval = [&](size_t claim, size_t column) {
    return column < cw[claim].size() ? out.powers[claim] * cw[claim][column] : F::zero();
  };
  for (size_t k = 0; k < log_cols; ++k) {
    size_t half = logical / 2;
    F lc = F::zero(), rc = F::zero();
    for (size_t col = 0; col < half; ++col)
      for (size_t i = 0; i < claims.size(); ++i) {
        F lower = eval_at(col, i), upper = eval_at(col + half, i);
        lc += lower * wval(i, col + half);
        rc += upper * wval(i, col);
      }
    t.push_response(lc);
    t.push_response(rc);
    F ch = t.challenge_nonzero("multi-eval-fold");
    F inv = ch.inverse();
    out.rhs += lc * ch + rc * inv;
    // matrix.fold_columns(inv)
    {
      std::vector<std::vector<std::pair<size_t, F>>> upper;
      if (terms.size() > half) { upper.assign(terms.begin() + half, terms.end()); terms.resize(half); }
      for (size_t idx = 0; idx < upper.size(); ++idx) {
        if (idx == terms.size()) terms.emplace_back();
        for (const auto& [src, coef] : upper[idx]) terms[idx].push_back({src, coef * inv});
      }
    }
    // weights.fold_columns(ch)
    for (auto& w : cw) {
      std::vector<F> up;
      if (w.size() > half) { up.assign(w.begin() + half, w.end()); w.resize(half); }
      for (size_t idx = 0; idx < up.size(); ++idx) {
        if (idx == w.size()) w.push_back(F::zero());
        w[idx] += up[idx] * ch;
      }
    }
    logical = half;
    out.a_point.push_back(inv);
    out.b_point.push_back(ch);
  }
  for (size_t i = 0; i < claims.size(); ++i) out.row_scale.push_back(out.powers[i] * cw[i][0]);
  if (!terms.empty()) out.terms0 = terms[0];
  return out;
}

template <class F>
void validate_multi_eval(const std::vector<EvalClaim<F>>& claims, size_t real, size_t log_rows, size_t log_cols) {
  const size_t cols = size_t(1) << log_cols;
  for (const auto& c : claims)
    if (c.row_point.size() != log_rows || c.col_weight.empty() || c.col_weight.size() > cols)
      fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "multi-eval claim");
  if (claims.empty() || real == 0 || real > cols) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "multi-eval columns");
}

// `columns` are the real columns (setup alphas first, then the carry column),
// each of exactly `rows` entries (prove_multi_eval, qafold_short_decide.rs:466-536).
template <class F>
MultiEvalOut<F> prove_multi_eval(const std::vector<EvalClaim<F>>& claims, const std::vector<const std::vector<F>*>& columns,
                                 size_t log_rows, size_t log_cols, PcsTranscript<F>& t) {
  const size_t rows = size_t(1) << log_rows;
  const size_t real = columns.size();
  validate_multi_eval(claims, real, log_rows, log_cols);
  absorb_multi_eval_statement(claims, log_rows, log_cols, t);
  F rho = t.challenge_ext("multi-eval-batch");
  std::vector<std::vector<F>> row_w;
  for (const auto& c : claims) row_w.push_back(tensor_weights(c.row_point));
  // source evaluations[claim][source]
  std::vector<std::vector<F>> se(claims.size(), std::vector<F>(real, F::zero()));
  for (size_t i = 0; i < claims.size(); ++i)
#pragma omp parallel for if (rows >= 4096)
    for (long s = 0; s < long(real); ++s) {
      F acc = F::zero();
      const std::vector<F>& col = *columns[s];
      for (size_t r = 0; r < rows && r < col.size(); ++r) acc += row_w[i][r] * col[r];
      se[i][s] = acc;
    }
  MultiEvalColumns<F> mc = multi_eval_columns(claims, real, log_cols, rho, se, t);
  F rhs = mc.rhs;
  std::vector<F> a_point = mc.a_point, b_point = mc.b_point;
  std::vector<F> right(rows, F::zero());
  for (size_t i = 0; i < claims.size(); ++i) {
    F scale = mc.row_scale[i];
#pragma omp parallel for if (rows >= 4096)
    for (long r = 0; r < long(rows); ++r) right[r] += scale * row_w[i][r];
  }
  std::vector<F> folded(rows, F::zero());
#pragma omp parallel for if (rows >= 4096)
  for (long r = 0; r < long(rows); ++r) {
    F s = F::zero();
    for (const auto& [src, coef] : mc.terms0) {
      const std::vector<F>& col = *columns[src];
      if (size_t(r) < col.size()) s += col[r] * coef;
    }
    folded[r] = s;
  }
  std::vector<F> left = folded;
  for (size_t k = 0; k < log_rows; ++k) {
    size_t half = left.size() / 2;
    F lc = F::zero(), rc = F::zero();
    for (size_t i = 0; i < half; ++i) { lc += left[i] * right[half + i]; rc += left[half + i] * right[i]; }
    t.push_response(lc);
    t.push_response(rc);
    F ch = t.challenge_nonzero("multi-eval-fold");
    F inv = ch.inverse();
    rhs += lc * ch + rc * inv;
    for (size_t i = 0; i < half; ++i) { left[i] += left[half + i] * inv; right[i] += right[half + i] * ch; }
    left.resize(half);
    right.resize(half);
    a_point.push_back(inv);
    b_point.push_back(ch);
  }
  F a = left[0], b = right[0];
  t.push_response(a);
  t.push_response(b);
  F ew = expected_weight_eval(claims, mc.powers, log_cols, b_point);
  MultiEvalOut<F> out;
  out.ok = (a * b == rhs) && (b == ew);
  out.reduced = {a, a_point};
  out.folded_vector = std::move(folded);
  return out;
}

template <class F>
MultiEvalOut<F> verify_multi_eval(const std::vector<EvalClaim<F>>& claims, size_t log_rows, size_t log_cols, PcsTranscript<F>& t) {
  const size_t cols = size_t(1) << log_cols;
  for (const auto& c : claims)
    if (c.row_point.size() != log_rows || c.col_weight.empty() || c.col_weight.size() > cols)
      fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "multi-eval claim");
  if (claims.empty()) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "multi-eval claims");
  absorb_multi_eval_statement(claims, log_rows, log_cols, t);
  F rho = t.challenge_ext("multi-eval-batch");
  F rhs = F::zero(), power = F::one();
  std::vector<F> powers;
  for (const auto& c : claims) { powers.push_back(power); rhs += power * c.value; power *= rho; }
  std::vector<F> a_point, b_point;
  for (size_t k = 0; k < log_rows + log_cols; ++k) {
    F lc = t.read_response(), rc = t.read_response();
    F ch = t.challenge_nonzero("multi-eval-fold");
    F inv = ch.inverse();
    rhs += lc * ch + rc * inv;
    a_point.push_back(inv);
    b_point.push_back(ch);
  }
  F a = t.read_response(), b = t.read_response();
  F ew = expected_weight_eval(claims, powers, log_cols, b_point);
  MultiEvalOut<F> out;
  out.ok = (a * b == rhs) && (b == ew);
  out.reduced = {a, a_point};
  return out;
}

// ------------------------------------------------------------ transcript pieces
template <class F>
void absorb_selection(PcsTranscript<F>& t, const RowSelection& s) {
  if (s.all) {
    t.absorb_str("selection-kind", "all");
    t.absorb_u64("selection-count", s.count);
  } else {
    t.absorb_str("selection-kind", "partial");
    t.absorb_u64("selection-count", s.rows.size());
    for (size_t r : s.rows) t.absorb_u64("selection-row", r);
  }
}
template <class F>
void absorb_round_context(PcsTranscript<F>& t, size_t level, const SetupLevel<F>& sl, const std::optional<Digest>& carry) {
  t.absorb_str("decide-round-domain", "qafold-short/decide-round/v1");
  t.absorb_u64("decide-round-level", level);
  const SetupShape& s = sl.shape;
  t.absorb_u64("decide-round-shape-level", s.level);
  t.absorb_u64("decide-round-shape-encoded-rows", s.encoded_rows);
  t.absorb_u64("decide-round-shape-message-rows", s.message_rows);
  t.absorb_u64("decide-round-shape-t-cols", s.t_cols);
  t.absorb_u64("decide-round-shape-t-elements", s.t_elements);
  t.absorb_u64("decide-round-shape-t-last-len", s.t_last_len);
  t.absorb_u64("decide-round-shape-h-cols", s.h_cols);
  t.absorb_digest("decide-round-setup-root", sl.root);
  if (carry) { t.absorb_u8("decide-round-carry-present", 1); t.absorb_digest("decide-round-carry-root", *carry); }
  else t.absorb_u8("decide-round-carry-present", 0);
}
template <class F>
void absorb_next_carry(PcsTranscript<F>& t, const std::optional<Digest>& carry) {
  t.absorb_str("decide-next-carry-domain", "qafold-short/decide-next-carry/v1");
  if (carry) { t.absorb_u8("decide-next-carry-present", 1); t.absorb_digest("decide-next-carry-root", *carry); }
  else t.absorb_u8("decide-next-carry-present", 0);
}
template <class F>
void absorb_iota_statement(PcsTranscript<F>& t, size_t level, const SetupLevel<F>& sl, const std::optional<Digest>& carry,
                           size_t carry_cols, const RowSelection& sel, const std::vector<F>& col_weights) {
  t.absorb_str("iota-domain", "qafold-short/decide-iota/v1");
  t.absorb_u64("iota-level", level);
  const SetupShape& s = sl.shape;
  t.absorb_u64("iota-shape-level", s.level);
  t.absorb_u64("iota-shape-encoded-rows", s.encoded_rows);
  t.absorb_u64("iota-shape-message-rows", s.message_rows);
  t.absorb_u64("iota-shape-t-cols", s.t_cols);
  t.absorb_u64("iota-shape-t-elements", s.t_elements);
  t.absorb_u64("iota-shape-t-last-len", s.t_last_len);
  t.absorb_u64("iota-shape-h-cols", s.h_cols);
  t.absorb_digest("iota-setup-root", sl.root);
  if (carry) { t.absorb_u8("iota-carry-present", 1); t.absorb_digest("iota-carry-root", *carry); }
  else t.absorb_u8("iota-carry-present", 0);
  t.absorb_u64("iota-carry-cols", carry_cols);
  absorb_selection(t, sel);
  t.absorb_exts("iota-column-weights", col_weights);
}
template <class F>
void absorb_direct_switch(PcsTranscript<F>& t, const QaCode<F>& target, size_t target_level, size_t row_factor,
                          const RowSelection& sel, const std::vector<F>& iota, F merged_value, const std::vector<F>& merged_left) {
  t.absorb_str("direct-code-switch-domain", "qafold-short/decide-direct-code-switch/v2");
  t.absorb_u64("direct-code-switch-target-level", target_level);
  t.absorb_u64("direct-code-switch-row-factor", row_factor);
  t.absorb_u64("direct-code-switch-message-len", target.message_len);
  t.absorb_u64("direct-code-switch-encoded-len", target.codeword_len());
  t.absorb_u64("direct-code-switch-target-index", target.index);
  t.absorb_digest("direct-code-switch-target-generator", target.generator_digest);
  absorb_selection(t, sel);
  t.absorb_exts("direct-code-switch-iota", iota);
  t.absorb_ext("direct-code-switch-merged-value", merged_value);
  t.absorb_exts("direct-code-switch-merged-left-point", merged_left);
}
template <class F>
void absorb_opening_statement(PcsTranscript<F>& t, const PcsParams<F>& pp, const Reduction<F>& red) {
  t.absorb_str("decide-domain", "qafold-short/decide/v1");
  t.absorb_digest("decide-parameters", pp.parameter_digest);
  t.absorb_digest("decide-setup", pp.setup_digest);
  t.absorb_u64("decide-levels", pp.levels());
  t.absorb_u8("opening-reduction-ok", red.ok ? 1 : 0);
  t.absorb_u64("pending-h-count", red.pending.size());
  for (const auto& p : red.pending) {
    t.absorb_u64("pending-h-level", p.level);
    t.absorb_ext("pending-g-value", p.value);
    t.absorb_exts("pending-g-left", p.left_point);
    t.absorb_exts("pending-g-right", p.right_point);
  }
}

template <class F>
std::vector<std::vector<MatrixClaim<F>>> prepare_pending_h(const PcsParams<F>& pp, const Reduction<F>& red, PcsTranscript<F>& t) {
  const size_t L = pp.levels();
  if (!red.ok || red.pending.size() != (L > 0 ? L - 1 : 0)) fail(QF_E_INVALID_COMMITMENT, "pending order");
  for (size_t i = 0; i < red.pending.size(); ++i)
    if (red.pending[i].level != L - 1 - i) fail(QF_E_INVALID_COMMITMENT, "pending level");
  absorb_opening_statement(t, pp, red);
  std::vector<std::vector<MatrixClaim<F>>> by_level(L);
  for (const auto& p : red.pending) {
    const QaCode<F>& code = pp.seq.codes[p.level];
    by_level[p.level].push_back(reduce_generator_claim(code.message_len, code.index, MatrixClaim<F>{p.value, p.left_point, p.right_point}));
  }
  return by_level;
}

struct PreparedShape {
  size_t log_rows, log_cols, setup_cols, carry_cols;
};
template <class F>
std::vector<EvalClaim<F>> prepare_eval_claims(const PcsParams<F>& pp, size_t level, const std::vector<MatrixClaim<F>>& h,
                                              const std::optional<EvalWithPoint<F>>& w, PreparedShape& shape) {
  const QaCode<F>& code = pp.seq.codes[level];
  const QaCode<F>& target = pp.seq.codes[level - 1];
  const SetupLevel<F>& sl = pp.setup_level(level);
  const size_t rows = code.message_len, log_rows = ilog2(rows);
  sl.shape.validate();
  const size_t setup_cols = code.alphas.size();
  if (sl.shape.message_rows != target.message_len || sl.shape.encoded_rows != target.codeword_len() || sl.shape.t_cols != 0 ||
      sl.shape.h_cols != code.alphas.size() * pp.seq.switch_ratio || rows != target.message_len * pp.seq.switch_ratio)
    fail(QF_E_ENCODING, "decide claim shape");
  std::vector<EvalClaim<F>> claims;
  for (const auto& c : h) {
    if (c.left.size() != log_rows || c.right.size() != size_t(ilog2(code.alphas.size())))
      fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "h claim dims");
    claims.push_back({c.value, c.left, tensor_weights(c.right)});
  }
  size_t carry_cols = 0;
  if (w) {
    if (w->point.size() != log_rows) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "w claim dims");
    std::vector<F> cwt(setup_cols, F::zero());
    cwt.push_back(F::one());
    claims.push_back({w->value, w->point, cwt});
    carry_cols = 1;
  }
  if (claims.empty()) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "no decide claims");
  shape = {log_rows, size_t(ilog2(next_pow2(setup_cols + carry_cols))), setup_cols, carry_cols};
  return claims;
}

template <class F>
std::vector<F> iota_weights(const std::vector<F>& logical_w, size_t setup_cols, size_t carry_cols, const std::vector<F>& row_point,
                            size_t row_factor) {
  size_t block_log = ilog2(row_factor);
  std::vector<F> bw = tensor_weights(std::vector<F>(row_point.begin(), row_point.begin() + block_log));
  size_t logical = setup_cols + carry_cols;
  std::vector<F> pw(next_pow2(logical * row_factor), F::zero());
  for (size_t lc = 0; lc < logical; ++lc)
    for (size_t b = 0; b < row_factor; ++b) pw[lc * row_factor + b] = logical_w[lc] * bw[b];
  return pw;
}

// A direct-interleaved carry: one logical column split into `row_factor`
// physical columns and encoded with the next lower code.
template <class F>
struct Carry {
  std::vector<F> message;                // logical column
  std::unique_ptr<CodewordView<F>> cw;   // on the host, or kept on a device
};

template <class F>
F setup_row_value(const SetupRows<F>& rows, const SetupShape& shape, size_t ordinal, size_t row, const std::vector<F>& w) {
  const size_t tc = shape.total_cols();
  F s = F::zero();
  if (!rows.all) {
    const auto& q = rows.partial.at(ordinal);
    if (q.row_index != row || q.row.size() != tc) fail(QF_E_INVALID_COMMITMENT, "setup row");
    for (size_t c = 0; c < tc; ++c) s += w[c] * q.row[c];
  } else {
    for (size_t c = 0; c < tc; ++c) s += w[c] * rows.encoded[c * shape.encoded_rows + row];
  }
  return s;
}
template <class F>
F carry_row_value(const Rows<F>& rows, size_t n_enc, size_t n_cols, size_t ordinal, size_t row, const F* w) {
  F s = F::zero();
  if (!rows.all) {
    const auto& q = rows.partial.at(ordinal);
    if (q.row.size() != n_cols) fail(QF_E_INVALID_COMMITMENT, "carry row");
    for (size_t c = 0; c < n_cols; ++c) s += q.row[c] * w[c];
  } else {
    for (size_t c = 0; c < n_cols; ++c) s += w[c] * rows.encoded[c * n_enc + row];
  }
  return s;
}
// body(i) for i in [0, n) on the OpenMP threads when n >= min_n; the first
// exception any iteration throws is rethrown on the calling thread (none may
// leave a parallel region).
template <class Fn>
void parallel_rows(size_t n, size_t min_n, Fn&& body) {
  std::exception_ptr err;
  std::mutex mu;
#pragma omp parallel for if (n >= min_n) schedule(static)
  for (long i = 0; i < long(n); ++i) {
    try {
      body(size_t(i));
    } catch (...) {
      std::lock_guard<std::mutex> g(mu);
      if (!err) err = std::current_exception();
    }
  }
  if (err) std::rethrow_exception(err);
}

template <class F>
std::vector<F> compute_iota(const SetupLevel<F>& sl, const SetupRows<F>& srows, const std::optional<Rows<F>>& crows,
                            size_t carry_cols, const RowSelection& sel, const std::vector<F>& w) {
  const size_t tc = sl.shape.total_cols();
  std::vector<F> iota(sel.size());
  parallel_rows(sel.size(), 64, [&](size_t i) {
    size_t row = sel.at(i);
    F v = setup_row_value(srows, sl.shape, i, row, w);
    if (crows) v += carry_row_value(*crows, sl.shape.encoded_rows, carry_cols, i, row, w.data() + tc);
    iota[i] = v;
  });
  return iota;
}

template <class F>
SetupRows<F> open_setup_rows(const SetupLevel<F>& sl, const RowSelection& sel) {
  SetupRows<F> out;
  out.shape = sl.shape;
  if (sel.all) { out.all = true; out.encoded = sl.encoded; return out; }
  const size_t tc = sl.shape.total_cols();
  out.partial.resize(sel.rows.size());
  parallel_rows(sel.rows.size(), 64, [&](size_t i) {
    const size_t r = sel.rows[i];
    SetupRowQuery<F>& q = out.partial[i];
    q.row_index = r;
    q.row.resize(tc);
    for (size_t c = 0; c < tc; ++c) q.row[c] = sl.encoded[c * sl.shape.encoded_rows + r];
    q.path.siblings = sl.tree.path(r);
  });
  return out;
}
template <class F>
Rows<F> open_codeword_rows(const Codeword<F>& cw, const RowSelection& sel) {
  Rows<F> out;
  if (sel.all) { out.all = true; out.n_rows = cw.n_ext_rows; out.n_cols = cw.n_cols; out.encoded = cw.encoded; return out; }
  out.partial.resize(sel.rows.size());
  parallel_rows(sel.rows.size(), 64, [&](size_t i) {
    const size_t r = sel.rows[i];
    out.partial[i].row = cw.row(r);
    out.partial[i].path.siblings = cw.tree.path(r);
  });
  return out;
}
// The same rows of a codeword held anywhere (a device codeword gathers them).
template <class F>
Rows<F> open_codeword_rows(const CodewordView<F>& cw, const RowSelection& sel) {
  if (const auto* host = dynamic_cast<const Codeword<F>*>(&cw)) return open_codeword_rows(*host, sel);
  Rows<F> out;
  if (sel.all) { out.all = true; out.n_rows = cw.ext_rows(); out.n_cols = cw.cols(); out.encoded = cw.entries(); return out; }
  auto rows = cw.rows(sel.rows);
  auto paths = cw.paths(sel.rows);
  out.partial.resize(sel.rows.size());
  for (size_t i = 0; i < sel.rows.size(); ++i) {
    out.partial[i].row = std::move(rows[i]);
    out.partial[i].path.siblings = std::move(paths[i]);
  }
  return out;
}

template <class F>
struct SwitchCarry {
  MatrixClaim<F> generator_claim;
  EvalWithPoint<F> folded_w;
};

template <class F>
SwitchCarry<F> prove_direct_switch(const QaCode<F>& target, size_t target_level, size_t row_factor, const RowSelection& sel,
                                   const std::vector<F>& iota, const std::vector<F>& folded_message, F merged_value,
                                   const std::vector<F>& merged_left, PcsTranscript<F>& t) {
  size_t block_log = ilog2(row_factor);
  std::vector<F> base_point(merged_left.begin() + block_log, merged_left.end());
  if (folded_message.size() != target.message_len) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "switch message");
  F ev;
  if (!mle_eval(folded_message, base_point, ev) || ev != merged_value) fail(QF_E_INVALID_COMMITMENT, "switch merged value");
  absorb_direct_switch(t, target, target_level, row_factor, sel, iota, merged_value, merged_left);
  size_t sel_log = ilog2(next_pow2(sel.size()));
  std::vector<F> slp;
  for (size_t i = 0; i < sel_log; ++i) slp.push_back(t.challenge_ext("direct-code-switch-selection-left"));
  std::vector<F> sl = tensor_weights_prefix(slp, sel.size());
  F selected = inner_product(sl, iota);
  const size_t n_enc = target.codeword_len();
  std::vector<F> sparse(n_enc, F::zero());
  for (size_t i = 0; i < sel.size(); ++i) sparse[sel.at(i)] += sl[i];
  std::vector<F> gl = target.generator_left_projection(sparse);
  F rho = t.challenge_ext("direct-code-switch-opening-batch");
  std::vector<F> ml = tensor_weights(base_point);
  F combined = selected + rho * merged_value;
  for (size_t i = 0; i < gl.size(); ++i) gl[i] = gl[i] + rho * ml[i];
  LiteBullet<F> msg = prove_litebullet<F>(combined, std::move(gl), folded_message, t, "decide-direct-carry-message-litebullet");
  F ole = tensor_inner_product(base_point, msg.a_point);
  F sle = msg.a_value - rho * ole;
  std::vector<F> gr = target.generator_right_projection(tensor_weights(msg.a_point));
  LiteBullet<F> gen = prove_litebullet<F>(sle, std::move(sparse), std::move(gr), t, "decide-direct-carry-generator-litebullet");
  return {MatrixClaim<F>{gen.b_value, gen.b_point, msg.a_point}, EvalWithPoint<F>{msg.b_value, msg.b_point}};
}

template <class F>
std::optional<SwitchCarry<F>> verify_direct_switch(const QaCode<F>& target, size_t target_level, size_t row_factor,
                                                   const RowSelection& sel, const std::vector<F>& iota, F merged_value,
                                                   const std::vector<F>& merged_left, PcsTranscript<F>& t) {
  absorb_direct_switch(t, target, target_level, row_factor, sel, iota, merged_value, merged_left);
  size_t block_log = ilog2(row_factor);
  std::vector<F> base_point(merged_left.begin() + block_log, merged_left.end());
  size_t sel_log = ilog2(next_pow2(sel.size()));
  std::vector<F> slp;
  for (size_t i = 0; i < sel_log; ++i) slp.push_back(t.challenge_ext("direct-code-switch-selection-left"));
  std::vector<F> sl = tensor_weights_prefix(slp, sel.size());
  F selected = inner_product(sl, iota);
  F rho = t.challenge_ext("direct-code-switch-opening-batch");
  F combined = selected + rho * merged_value;
  auto msg = verify_litebullet<F>(combined, target.message_len, t, "decide-direct-carry-message-litebullet");
  if (!msg) return std::nullopt;
  F ole = tensor_inner_product(base_point, msg->a_point);
  F sle = msg->a_value - rho * ole;
  auto gen = verify_litebullet<F>(sle, target.codeword_len(), t, "decide-direct-carry-generator-litebullet");
  if (!gen) return std::nullopt;
  F expected = F::zero();
  for (size_t i = 0; i < sel.size(); ++i) expected += sl[i] * tensor_weight_at(gen->a_point, sel.at(i));
  if (gen->a_value != expected) return std::nullopt;
  return SwitchCarry<F>{MatrixClaim<F>{gen->b_value, gen->b_point, msg->a_point}, EvalWithPoint<F>{msg->b_value, msg->b_point}};
}

// ------------------------------------------------------------ prove / verify
// Runs a MultiEval over one level's alpha columns, plus the carried message
// as the last column when `carry_message` is given, with the row vectors on
// a device.  Same transcript as prove_multi_eval; `folded_vector` is returned
// already block-folded at the reduced point's first log2(row_factor)
// coordinates (fold_short_direct_interleaved_witness), i.e. rows / row_factor
// entries.  Returns false, before touching the transcript, to leave a small
// MultiEval on the host.
template <class F>
struct DecideAccel {
  virtual ~DecideAccel() {}
  virtual bool multi_eval(const PcsParams<F>& pp, size_t level, const std::vector<EvalClaim<F>>& claims,
                          const std::vector<F>* carry_message, size_t log_rows, size_t log_cols, size_t row_factor,
                          PcsTranscript<F>& t, MultiEvalOut<F>& out) = 0;
  // prove_direct_switch with its message-length vectors on the device;
  // returns false to keep the (small) switch on the host.
  virtual bool direct_switch(const QaCode<F>& target, size_t target_level, size_t row_factor, const RowSelection& sel,
                             const std::vector<F>& iota, const std::vector<F>& folded_message, F merged_value,
                             const std::vector<F>& merged_left, PcsTranscript<F>& t, SwitchCarry<F>& out) {
    return false;
  }
  // The carry commitment (commit_extension_matrix of `message` under
  // pp.seq.codes[code_index], `n_cols` columns, extension-row leaves) kept on
  // the device; null leaves it to the host.
  virtual std::unique_ptr<CodewordView<F>> commit_carry(const PcsParams<F>& pp, size_t code_index,
                                                        const std::vector<F>& message, size_t n_cols) {
    return nullptr;
  }
};

template <class F>
DecideProof<F> prove_decide(const PcsParams<F>& pp, const Reduction<F>& red, DecideAccel<F>* accel = nullptr) {
  const size_t L = pp.levels();
  PcsTranscript<F> t;
  std::vector<std::vector<MatrixClaim<F>>> h;
  {
    Section sec("decide_pending_h");
    h = prepare_pending_h(pp, red, t);
  }
  DecideProof<F> proof;
  if (L <= 1) {
    for (auto& v : h) if (!v.empty()) fail(QF_E_INVALID_COMMITMENT, "base-level claims");
    proof.responses = std::move(t.responses);
    return proof;
  }
  std::optional<EvalWithPoint<F>> w_claim;
  std::unique_ptr<Carry<F>> carry;
  std::optional<Digest> carry_root;
  const size_t rf = pp.seq.switch_ratio;
  for (size_t level = L - 1; level >= 1; --level) {
    const SetupLevel<F>& sl = pp.setup_level(level);
    std::vector<MatrixClaim<F>> lh = std::move(h[level]);
    h[level].clear();
    PreparedShape ps;
    std::vector<EvalClaim<F>> claims = prepare_eval_claims(pp, level, lh, w_claim, ps);
    if ((carry != nullptr) != (ps.carry_cols > 0) || (carry != nullptr) != carry_root.has_value())
      fail(QF_E_INVALID_COMMITMENT, "carry presence");
    absorb_round_context(t, level, sl, carry_root);
    const QaCode<F>& code = pp.seq.codes[level];
    std::vector<const std::vector<F>*> cols;
    for (const auto& a : code.alphas) cols.push_back(&a);
    if (carry) cols.push_back(&carry->message);
    MultiEvalOut<F> me;
    const bool on_device = accel && accel->multi_eval(pp, level, claims, carry ? &carry->message : nullptr, ps.log_rows,
                                                      ps.log_cols, pp.seq.switch_ratio, t, me);
    if (!on_device) {
      Section sec("decide_multi_eval_host");
      me = prove_multi_eval(claims, cols, ps.log_rows, ps.log_cols, t);
    }
    if (!me.ok || me.reduced.point.size() != ps.log_cols + ps.log_rows) fail(QF_E_INVALID_COMMITMENT, "multi-eval");
    std::vector<F> col_point(me.reduced.point.begin(), me.reduced.point.begin() + ps.log_cols);
    std::vector<F> merged_left(me.reduced.point.begin() + ps.log_cols, me.reduced.point.end());
    std::vector<F> col_w = tensor_weights(col_point);
    const QaCode<F>& target = pp.seq.codes[level - 1];
    const size_t n_enc = target.codeword_len();
    if (sl.shape.encoded_rows != n_enc) fail(QF_E_ENCODING, "setup rows");
    size_t qc = target.num_queries(pp.security_bits, n_enc, pp.card_log2);
    Digest seed = t.challenge_digest("decide-row-selection");
    RowSelection sel = make_selection(qc, n_enc, seed);
    DecideRound<F> round;
    round.level = level;
    {
      Section sec("decide_open_rows");
      round.setup_rows = open_setup_rows(sl, sel);
      if (carry) round.carry_rows = open_codeword_rows(*carry->cw, sel);
    }
    std::vector<F> iw = iota_weights(col_w, ps.setup_cols, ps.carry_cols, merged_left, rf);
    size_t auth_carry_cols = ps.carry_cols * rf;
    if (iw.size() != next_pow2(sl.shape.total_cols() + auth_carry_cols)) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "iota weights");
    absorb_iota_statement(t, level, sl, carry_root, auth_carry_cols, sel, iw);
    std::vector<F> iota;
    {
      Section sec("decide_iota");
      iota = compute_iota(sl, round.setup_rows, round.carry_rows, auth_carry_cols, sel, iw);
    }
    for (const F& v : iota) t.push_response(v);
    // Fold the block coordinate of the logical witness.
    const size_t trows = target.message_len;
    std::vector<F> recursive;
    if (on_device) {
      recursive = std::move(me.folded_vector);
    } else {
      std::vector<F> bw = tensor_weights(std::vector<F>(merged_left.begin(), merged_left.begin() + ilog2(rf)));
      recursive.assign(trows, F::zero());
      for (size_t r = 0; r < trows; ++r) {
        F s = F::zero();
        for (size_t b = 0; b < rf; ++b) s += me.folded_vector[b * trows + r] * bw[b];
        recursive[r] = s;
      }
    }
    if (recursive.size() != trows) fail(QF_E_ENCODING, "recursive witness length");
    std::unique_ptr<Carry<F>> next_carry;
    std::optional<Digest> next_root;
    std::vector<F> terminal;
    if (level > 1) {
      const QaCode<F>& nt = pp.seq.codes[level - 2];
      if (trows != nt.message_len * rf) fail(QF_E_ENCODING, "carry rows");
      next_carry = std::make_unique<Carry<F>>();
      next_carry->message = recursive;
      Section sec("decide_carry_commit");
      if (accel) next_carry->cw = accel->commit_carry(pp, level - 2, recursive, rf);
      if (!next_carry->cw) next_carry->cw = std::make_unique<Codeword<F>>(encode_and_commit(nt, recursive, rf, kLeafExtDomain));
      next_root = next_carry->cw->root();
    } else {
      terminal = recursive;
    }
    absorb_next_carry(t, next_root);
    const std::vector<F>& folded_for_switch = next_carry ? next_carry->message : terminal;
    SwitchCarry<F> sc;
    if (!(accel && accel->direct_switch(target, level - 1, rf, sel, iota, folded_for_switch, me.reduced.value, merged_left, t, sc))) {
      Section sec("decide_switch_host");
      sc = prove_direct_switch(target, level - 1, rf, sel, iota, folded_for_switch, me.reduced.value, merged_left, t);
    }
    if (level > 1) {
      h[level - 1].push_back(reduce_generator_claim(target.message_len, target.index, sc.generator_claim));
      w_claim = sc.folded_w;
      carry = std::move(next_carry);
      carry_root = next_root;
    } else {
      F ev;
      if (evaluate_generator_mle(target, sc.generator_claim.left, sc.generator_claim.right) != sc.generator_claim.value ||
          !mle_eval(terminal, sc.folded_w.point, ev) || ev != sc.folded_w.value)
        fail(QF_E_INVALID_COMMITMENT, "decide terminal");
      for (const F& v : terminal) t.push_response(v);
      proof.base_vector = terminal;
      carry.reset();
      carry_root.reset();
    }
    round.next_carry_root = next_root;
    proof.rounds.push_back(std::move(round));
  }
  for (auto& v : h) if (!v.empty()) fail(QF_E_INVALID_COMMITMENT, "unconsumed claims");
  proof.responses = std::move(t.responses);
  return proof;
}

template <class F>
bool verify_setup_rows(const SetupLevel<F>& sl, const RowSelection& sel, const SetupRows<F>& rows) {
  const SetupShape& s = sl.shape;
  if (sel.all != rows.all) return false;
  if (rows.all) {
    if (sel.count != s.encoded_rows || !(rows.shape == s) || rows.encoded.size() != s.encoded_rows * s.total_cols()) return false;
    return build_setup_tree<F>(rows.encoded, s).root() == sl.root;
  }
  if (rows.partial.size() != sel.rows.size()) return false;
  for (size_t i = 0; i < rows.partial.size(); ++i) {
    const auto& q = rows.partial[i];
    if (q.row_index != sel.rows[i] || q.row.size() != s.total_cols()) return false;
    Digest leaf = hash_setup_row<F>(q.row.data(), s, q.row_index);
    if (!verify_merkle_siblings(leaf, q.row_index, s.encoded_rows, q.path.siblings, sl.root)) return false;
  }
  return true;
}
template <class F>
bool verify_carry_rows(const Digest& root, size_t n_enc, size_t n_cols, const RowSelection& sel, const Rows<F>& rows) {
  if (sel.all != rows.all) return false;
  if (rows.all) {
    if (sel.count != n_enc || rows.n_rows != n_enc || rows.n_cols != n_cols || rows.encoded.size() != n_enc * n_cols) return false;
    return build_row_tree<F>(kLeafExtDomain, rows.encoded, n_enc, n_cols).root() == root;
  }
  if (rows.partial.size() != sel.rows.size()) return false;
  for (size_t i = 0; i < rows.partial.size(); ++i) {
    const auto& q = rows.partial[i];
    if (q.row.size() != n_cols) return false;
    Digest leaf = hash_row<F>(kLeafExtDomain, q.row.data(), n_cols);
    if (!verify_merkle_siblings(leaf, sel.rows[i], n_enc, q.path.siblings, root)) return false;
  }
  return true;
}

template <class F>
bool verify_decide(const PcsParams<F>& pp, const Reduction<F>& red, const DecideProof<F>& proof) {
  if (!red.ok) return false;
  const size_t L = pp.levels();
  PcsTranscript<F> t(&proof.responses);
  auto h = prepare_pending_h(pp, red, t);
  if (L <= 1) {
    for (auto& v : h) if (!v.empty()) return false;
    return proof.rounds.empty() && proof.base_vector.empty() && t.exhausted();
  }
  if (proof.rounds.size() != L - 1) return false;
  std::optional<EvalWithPoint<F>> w_claim;
  std::optional<Digest> carry_root;
  const size_t rf = pp.seq.switch_ratio;
  size_t ri = 0;
  for (size_t level = L - 1; level >= 1; --level, ++ri) {
    const DecideRound<F>& round = proof.rounds[ri];
    if (round.level != level) return false;
    const SetupLevel<F>& sl = pp.setup_level(level);
    std::vector<MatrixClaim<F>> lh = std::move(h[level]);
    h[level].clear();
    PreparedShape ps;
    std::vector<EvalClaim<F>> claims = prepare_eval_claims(pp, level, lh, w_claim, ps);
    if (carry_root.has_value() != (ps.carry_cols > 0)) return false;
    absorb_round_context(t, level, sl, carry_root);
    MultiEvalOut<F> me = verify_multi_eval(claims, ps.log_rows, ps.log_cols, t);
    if (!me.ok || me.reduced.point.size() != ps.log_cols + ps.log_rows) return false;
    std::vector<F> col_point(me.reduced.point.begin(), me.reduced.point.begin() + ps.log_cols);
    std::vector<F> merged_left(me.reduced.point.begin() + ps.log_cols, me.reduced.point.end());
    std::vector<F> col_w = tensor_weights(col_point);
    const QaCode<F>& target = pp.seq.codes[level - 1];
    const size_t n_enc = target.codeword_len();
    size_t qc = target.num_queries(pp.security_bits, n_enc, pp.card_log2);
    Digest seed = t.challenge_digest("decide-row-selection");
    RowSelection sel = make_selection(qc, n_enc, seed);
    std::vector<F> iw = iota_weights(col_w, ps.setup_cols, ps.carry_cols, merged_left, rf);
    size_t auth_carry_cols = ps.carry_cols * rf;
    if ((round.carry_rows.has_value()) != (auth_carry_cols > 0)) return false;
    if (!verify_setup_rows(sl, sel, round.setup_rows)) return false;
    if (carry_root && !verify_carry_rows(*carry_root, n_enc, auth_carry_cols, sel, *round.carry_rows)) return false;
    absorb_iota_statement(t, level, sl, carry_root, auth_carry_cols, sel, iw);
    std::vector<F> iota;
    try {
      iota = compute_iota(sl, round.setup_rows, round.carry_rows, auth_carry_cols, sel, iw);
    } catch (const QfError&) {
      return false;
    }
    for (const F& v : iota)
      if (t.read_response() != v) return false;
    std::optional<Digest> next_root;
    if (level > 1) {
      if (!round.next_carry_root) return false;
      next_root = round.next_carry_root;
    } else if (round.next_carry_root) {
      return false;
    }
    absorb_next_carry(t, next_root);
    auto sc = verify_direct_switch(target, level - 1, rf, sel, iota, me.reduced.value, merged_left, t);
    if (!sc) return false;
    if (level > 1) {
      h[level - 1].push_back(reduce_generator_claim(target.message_len, target.index, sc->generator_claim));
      w_claim = sc->folded_w;
      carry_root = next_root;
    } else {
      if (evaluate_generator_mle(target, sc->generator_claim.left, sc->generator_claim.right) != sc->generator_claim.value ||
          proof.base_vector.size() != target.message_len)
        return false;
      for (const F& v : proof.base_vector)
        if (t.read_response() != v) return false;
      F ev;
      if (!mle_eval(proof.base_vector, sc->folded_w.point, ev) || ev != sc->folded_w.value) return false;
      carry_root.reset();
    }
  }
  for (auto& v : h) if (!v.empty()) return false;
  return !carry_root && t.exhausted();
}

}  // namespace qf
