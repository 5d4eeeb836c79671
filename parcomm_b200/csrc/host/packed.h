// Packed PCS: `lanes` base values per extension element, Boolean-to-monomial
// (Mobius) transform, QAFold commitment, and the authenticated Boolean-MLE
// openings (single block and the block-axis batch).
//
// Reference: packed.rs:132-779 (PackedPcs::new/commit/open/verify,
// equality_table, project_lanes, apply_weight_images, round_message,
// fold_pair, batch_weight, mobius_in_place, Transcript) and packed_batch.rs
// (open_batch_impl 139-319, verify_batch 321-422); codeword-fold binding
// qafold_short_batch.rs:59-240.
//
// The heavy data-parallel steps are delegated to a `Backend` (the CUDA
// implementation in the product library; a plain CPU restatement in the
// oracle).  Everything here is sequential protocol logic.
#pragma once
#include <map>
#include <mutex>
#include <tuple>
#include <chrono>
#include <functional>
#include <memory>

#include "decide.h"

namespace qf {

// ------------------------------------------------------------ packed transcript
template <class F>
struct PackedTranscript {
  Blake2s h;
  void bytes(const void* p, size_t n) { h.update_u64(n); h.update(p, n); }
  void bytes_str(const char* s) { bytes(s, std::strlen(s)); }
  void field(const F& v) { uint8_t e[F::kBytes]; v.to_bytes(e); bytes(e, F::kBytes); }
  F challenge() {
    for (uint64_t counter = 0;; ++counter) {
      Blake2s c = h;
      c.update_str("challenge");
      c.update_u64(counter);
      Digest d = c.finalize();
      F v;
      if (F::from_uniform_bytes(d.data(), v)) { bytes(d.data(), 32); return v; }
    }
  }
  F nonzero_challenge() { for (;;) { F v = challenge(); if (!v.is_zero()) return v; } }
};

template <class F>
std::vector<F> equality_table(const std::vector<F>& point) {
  std::vector<F> t(1, F::one());
  for (const F& c : point) {
    std::vector<F> n(t.size() * 2);
#pragma omp parallel for if (t.size() >= 4096)
    for (long i = 0; i < long(t.size()); ++i) { n[2 * i + 1] = t[i] * c; n[2 * i] = t[i] - n[2 * i + 1]; }
    t.swap(n);
  }
  return t;
}
template <class F>
F basis(int j) { F r = F::zero(); r.c[j] = 1; return r; }
template <class F>
std::vector<F> consecutive_powers(F v, size_t n) {
  std::vector<F> out;
  F p = F::one();
  for (size_t i = 0; i < n; ++i) { out.push_back(p); p = p * v; }
  return out;
}
// conjugates (packed_batch.rs:48-55): image -> sum_lane X^lane * Frob^{(L-image)}(lane value)
template <class F>
std::vector<F> conjugates(const std::vector<F>& lanes) {
  const int L = F::kLanes;
  std::vector<F> out(L);
  for (int image = 0; image < L; ++image) {
    F s = F::zero();
    for (int lane = 0; lane < L; ++lane) s += basis<F>(lane) * lanes[lane].frobenius((L - image) % L);
    out[image] = s;
  }
  return out;
}
// projected_claim (packed.rs:470-492): inverse DFT of the conjugate images
// recovers each lane MLE, then the low equality weights combine them.
template <class F>
F projected_claim(const std::vector<F>& evaluations, const std::vector<F>& low) {
  const int L = F::kLanes;
  F theta_inv = basis<F>(1).inverse();
  std::vector<F> inv_basis = consecutive_powers(theta_inv, L);
  uint32_t omega_inv = F::root_of_unity_inverse();
  uint32_t inv_l = F::base_inv(uint32_t(L));
  std::vector<F> conj(L);
  for (int i = 0; i < L; ++i) conj[i] = evaluations[i].frobenius(i);
  uint32_t omega_step = 1;
  F claim = F::zero();
  for (int j = 0; j < L; ++j) {
    uint32_t phase = 1;
    F sum = F::zero();
    for (int i = 0; i < L; ++i) { sum += conj[i].mul_prime(phase); phase = F::base_mul(phase, omega_step); }
    F lane = (sum * inv_basis[j]).mul_prime(inv_l);
    claim += low[j] * lane;
    omega_step = F::base_mul(omega_step, omega_inv);
  }
  return claim;
}
template <class F>
F round_evaluation(F claim, const F m[2], F ch) {
  F linear = claim - m[0] - m[0] - m[1];
  return m[0] + ch * (linear + ch * m[1]);
}
template <class F>
F batch_weight(const std::vector<F>& point, const std::vector<F>& reduced, const std::vector<F>& powers) {
  const int L = F::kLanes;
  F sum = F::zero();
  for (int i = 0; i < L; ++i) {
    F w = F::one();
    for (size_t k = 0; k < point.size(); ++k) {
      F s = point[k].frobenius((L - i) % L);
      w = w * ((F::one() - s) * (F::one() - reduced[k]) + s * reduced[k]);
    }
    sum += powers[i] * w;
  }
  return sum;
}
// folded_coefficients (packed_batch.rs:78-89)
template <class F>
std::vector<F> folded_coefficients(const std::vector<F>& high, const std::vector<F>& powers, F ch) {
  const int L = F::kLanes;
  std::vector<F> fwd = consecutive_powers(ch, high.size());
  std::vector<F> out(L);
  for (int image = 0; image < L; ++image) {
    F s = F::zero();
    for (size_t b = 0; b < high.size(); ++b) s += fwd[b] * high[b].frobenius((L - image) % L);
    out[image] = powers[image] * s;
  }
  return out;
}
// images[lane] = sum_image coefficients[image] * Frob^{(L-image)}(X^lane)
template <class F>
std::vector<F> weight_images(const std::vector<F>& coefficients) {
  const int L = F::kLanes;
  std::vector<F> images(L);
  for (int lane = 0; lane < L; ++lane) {
    F s = F::zero();
    for (int image = 0; image < L; ++image) s += coefficients[image] * basis<F>(lane).frobenius((L - image) % L);
    images[lane] = s;
  }
  return images;
}

// ------------------------------------------------------------ backend
struct StageTimes {
  double projection_ms = 0, folding_ms = 0, sumcheck_ms = 0, binding_ms = 0, native_opening_ms = 0, decide_ms = 0;
};

// Device- or host-resident heavy state for one packed PCS over a BVA.
template <class F>
struct Backend {
  virtual ~Backend() {}
  // Commit block `b` of the resident weights; keeps its codeword for openings.
  virtual Digest commit_block(size_t b) = 0;
  // Weights <- eq(outer); returns per-block lane projections (blocks x lanes).
  virtual std::vector<std::vector<F>> project_blocks(const std::vector<F>& outer, size_t blocks) = 0;
  // weights <- image map applied to the resident equality weights.
  virtual void apply_images(const std::vector<F>& images) = 0;
  // values <- sum_b fold[b] * packed(b, .); folded commit; returns its root.
  virtual Digest fold_and_commit(const std::vector<F>& fold_weights) = 0;
  // Degree-2 sumcheck round on (values, weights); fold with the challenge.
  virtual void sumcheck_message(F m[2]) = 0;
  virtual void sumcheck_fold(F ch) = 0;
  virtual F sumcheck_final_value() = 0;
  virtual F sumcheck_final_weight() = 0;
  // Binding payload for the sampled rows of every block and the folded codeword.
  virtual std::vector<uint8_t> binding_rows(const RowSelection& sel, const std::vector<Digest>& roots) = 0;
  // The folded codeword, for the native opening.
  virtual const CodewordView<F>& folded_codeword() = 0;
  // Top row projection of the folded codeword at tensor_weights(point[col_log..]);
  // a host backend also returns that row-weight vector in `row_weights`.
  virtual std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& row_weights) = 0;
  // Device execution of the folded codeword's top opening round, if any.
  virtual TopRoundAccel<F>* top_round_accel() { return nullptr; }
  // Device execution of the first Decide round, if any.
  virtual DecideAccel<F>* decide_accel() { return nullptr; }
};

// ------------------------------------------------------------ packed PCS
template <class F>
struct PackedPcs {
  size_t log_n = 0;  // base values per block, log2
  std::shared_ptr<PcsParams<F>> pp;
  size_t packed_len() const { return size_t(1) << (log_n - ilog2(F::kLanes)); }

  // The setup depends only on (log_n, columns, security bits, seed), so one
  // process builds each distinct setup once and shares it between parameter
  // sets (a pool of many shapes with few distinct block sizes).
  static PackedPcs create(size_t log_n, size_t columns, size_t security_bits, const std::array<uint8_t, 32>& seed,
                          SetupAccel<F>* accel = nullptr) {
    if (log_n < 4 || log_n > 30) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "packed log_n");
    static std::mutex mu;
    static std::map<std::tuple<size_t, size_t, size_t, std::array<uint8_t, 32>>, std::shared_ptr<PcsParams<F>>> cache;
    PackedPcs p;
    p.log_n = log_n;
    const auto key = std::make_tuple(log_n, columns, security_bits, seed);
    {
      std::lock_guard<std::mutex> g(mu);
      auto it = cache.find(key);
      if (it != cache.end()) {
        p.pp = it->second;
        return p;
      }
    }
    StdRng rng(seed);
    std::shared_ptr<PcsParams<F>> pp(
        pcs_setup<F>(size_t(1) << (log_n - ilog2(F::kLanes)), columns, security_bits, rng, accel).release());
    std::lock_guard<std::mutex> g(mu);
    p.pp = cache.emplace(key, pp).first->second;
    return p;
  }
  const Digest& parameter_digest() const { return pp->parameter_digest; }

  PackedTranscript<F> transcript(const Digest& root, const std::vector<F>& point, F value, const std::vector<uint8_t>& ctx) const {
    PackedTranscript<F> t;
    t.bytes_str(F::kPackedDomain);
    t.bytes(pp->parameter_digest.data(), 32);
    auto n = le64(log_n);
    t.bytes(n.data(), 8);
    t.bytes(root.data(), 32);
    t.bytes(ctx.data(), ctx.size());
    for (const F& c : point) t.field(c);
    t.field(value);
    return t;
  }
  PackedTranscript<F> batch_transcript(const std::vector<Digest>& roots, const std::vector<F>& point, F value,
                                       const std::vector<uint8_t>& ctx) const {
    PackedTranscript<F> t = transcript(roots[0], point, value, ctx);
    t.bytes_str("one-opening-block-packed-eo/v1");
    auto n = le64(roots.size());
    t.bytes(n.data(), 8);
    for (const auto& r : roots) t.bytes(r.data(), 32);
    return t;
  }
};

template <class F>
struct BatchOpening {
  F claimed_value;
  std::vector<uint8_t> wire;
  StageTimes times;
};

inline double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// open_batch_impl (packed_batch.rs:139-319) over the backend's resident blocks.
template <class F>
BatchOpening<F> open_batch(const PackedPcs<F>& pcs, Backend<F>& be, const std::vector<Digest>& roots, const std::vector<F>& point,
                           const std::vector<uint8_t>& ctx) {
  const int L = F::kLanes;
  const size_t lane_log = ilog2(L);
  const size_t blocks = roots.size();
  if (blocks < 2 || blocks > 128 || !is_pow2(blocks) || point.size() != pcs.log_n + ilog2(blocks))
    fail(QF_E_INVALID_PARAMETERS, "batched opening dimensions/profile");
  BatchOpening<F> out;
  auto t0 = std::chrono::steady_clock::now();
  const size_t split = ilog2(blocks);
  std::vector<F> outer(point.begin() + split, point.end() - lane_log);
  std::vector<F> low = equality_table(std::vector<F>(point.end() - lane_log, point.end()));
  std::vector<F> high = equality_table(std::vector<F>(point.begin(), point.begin() + split));
  std::vector<std::vector<F>> lanes = be.project_blocks(outer, blocks);
  std::vector<std::vector<F>> ev_by_block(blocks);
  for (size_t b = 0; b < blocks; ++b) ev_by_block[b] = conjugates(lanes[b]);
  std::vector<F> evaluations(L, F::zero());
  for (int image = 0; image < L; ++image)
    for (size_t b = 0; b < blocks; ++b) evaluations[image] += high[b].frobenius((L - image) % L) * ev_by_block[b][image];
  F claimed = projected_claim(evaluations, low);
  PackedTranscript<F> t = pcs.batch_transcript(roots, point, claimed, ctx);
  for (const F& v : evaluations) t.field(v);
  std::vector<F> powers = consecutive_powers(t.challenge(), L);
  F claim = F::zero();
  for (int i = 0; i < L; ++i) claim += powers[i] * evaluations[i];
  auto cross = [&](size_t witness, size_t query) {
    F s = F::zero();
    for (int image = 0; image < L; ++image) s += powers[image] * high[query].frobenius((L - image) % L) * ev_by_block[witness][image];
    return s;
  };
  std::vector<F> positive, negative;
  for (size_t d = 1; d < blocks; ++d) {
    F s = F::zero();
    for (size_t b = 0; b + d < blocks; ++b) s += cross(b, b + d);
    positive.push_back(s);
  }
  for (size_t d = 1; d < blocks; ++d) {
    F s = F::zero();
    for (size_t b = 0; b + d < blocks; ++b) s += cross(b + d, b);
    negative.push_back(s);
  }
  t.bytes_str("block-packed-eo-cross");
  for (const F& v : positive) t.field(v);
  for (const F& v : negative) t.field(v);
  F ch = t.nonzero_challenge();
  {
    F inv = ch.inverse(), fwd = ch, bwd = inv;
    for (size_t i = 0; i < positive.size(); ++i) { claim += positive[i] * fwd + negative[i] * bwd; fwd *= ch; bwd *= inv; }
  }
  std::vector<F> fold_weights = consecutive_powers(ch.inverse(), blocks);
  std::vector<F> coefficients = folded_coefficients(high, powers, ch);
  be.apply_images(weight_images(coefficients));
  out.times.projection_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  Digest folded_root = be.fold_and_commit(fold_weights);
  t.bytes(folded_root.data(), 32);
  out.times.folding_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  std::vector<std::array<F, 2>> rounds;
  std::vector<F> reduced;
  for (size_t k = 0; k < outer.size(); ++k) {
    F m[2];
    be.sumcheck_message(m);
    t.field(m[0]);
    t.field(m[1]);
    F c = t.challenge();
    claim = round_evaluation(claim, m, c);
    be.sumcheck_fold(c);
    rounds.push_back({m[0], m[1]});
    reduced.push_back(c);
  }
  F final_value = be.sumcheck_final_value();
  F final_weight = batch_weight(outer, reduced, coefficients);
  if (be.sumcheck_final_weight() != final_weight || claim != final_value * final_weight)
    fail(QF_E_INVALID_COMMITMENT, "batch sumcheck terminal");
  out.times.sumcheck_ms = ms_since(t0);
  // binding_seed (packed_batch.rs:94-98)
  t.bytes_str("authenticated-codeword-fold-queries/v1");
  t.field(final_value);
  Digest seed = t.h.finalize();
  t0 = std::chrono::steady_clock::now();
  const size_t rows = pcs.pp->top_ext_rows();
  size_t count = pcs.pp->num_queries(pcs.pp->levels() - 1, rows);
  RowSelection sel = make_selection(count, rows, seed);
  std::vector<uint8_t> binding = be.binding_rows(sel, roots);
  out.times.binding_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  const CodewordView<F>& folded = be.folded_codeword();
  const size_t col_log = ilog2(pcs.pp->extension_columns);
  std::vector<F> rw;
  std::vector<F> opening_vec = be.folded_opening(reduced, col_log, rw);
  F actual = inner_product(opening_vec, tensor_weights(std::vector<F>(reduced.begin(), reduced.begin() + col_log)));
  OpenResult<F> op = open_with_reduction(*pcs.pp, folded, reduced, opening_vec, actual, rw, be.top_round_accel());
  if (op.claimed != final_value || !op.reduction.ok) fail(QF_E_INVALID_COMMITMENT, "native opening value");
  out.times.native_opening_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  DecideProof<F> dp = prove_decide(*pcs.pp, op.reduction, be.decide_accel());
  out.times.decide_ms = ms_since(t0);
  const std::vector<uint8_t> ob = opening_to_bytes(op.proof);
  const std::vector<uint8_t> db = decide_to_bytes(dp);
  ByteWriter w;
  w.out.reserve(64 + (1 + evaluations.size() + positive.size() + negative.size() + 2 * rounds.size() + 1) * F::kBytes +
                binding.size() + ob.size() + db.size());
  w.bytes("QAPKBAT1", 8);
  w.field(claimed);
  for (const F& v : evaluations) w.field(v);
  for (const F& v : positive) w.field(v);
  for (const F& v : negative) w.field(v);
  w.digest(folded_root);
  for (const auto& m : rounds) { w.field(m[0]); w.field(m[1]); }
  w.field(final_value);
  w.len(binding.size());
  w.bytes(binding.data(), binding.size());
  w.len(ob.size());
  w.bytes(ob.data(), ob.size());
  w.len(db.size());
  w.bytes(db.data(), db.size());
  if (w.out.size() > 256u * 1024 * 1024) fail(QF_E_ENCODING, "oversize batch proof");
  out.claimed_value = claimed;
  out.wire = std::move(w.out);
  return out;
}

// Binding rows of one codeword (write_base_rows of the sampled payload).
template <class F>
void write_codeword_rows(ByteWriter& w, const Codeword<F>& cw, const RowSelection& sel) {
  Rows<F> r = open_codeword_rows(cw, sel);
  write_rows(w, r);
}

// verify_codeword_fold (qafold_short_batch.rs:162-240).
template <class F>
bool verify_codeword_fold(const PcsParams<F>& pp, const std::vector<Digest>& roots, const std::vector<F>& weights,
                          const Digest& folded, const Digest& seed, const uint8_t* bytes, size_t n) {
  const size_t rows = pp.top_ext_rows(), cols = pp.base_columns();
  if (roots.size() < 2 || roots.size() > 128 || !is_pow2(roots.size()) || roots.size() != weights.size()) return false;
  size_t count = pp.num_queries(pp.levels() - 1, rows);
  RowSelection sel = make_selection(count, rows, seed);
  ByteReader r(bytes, n);
  if (std::memcmp(r.take(8), "QAFOLDB1", 8) != 0 || r.len() != roots.size()) return false;
  std::vector<Rows<F>> payloads;
  for (size_t i = 0; i <= roots.size(); ++i) {
    const Digest& root = i < roots.size() ? roots[i] : folded;
    Rows<F> p = read_rows<F>(r);
    bool ok;
    if (!p.all) {
      ok = !sel.all && p.partial.size() == sel.size();
      for (size_t q = 0; ok && q < p.partial.size(); ++q) {
        if (p.partial[q].row.size() != cols) { ok = false; break; }
        Digest leaf = hash_row<F>(kLeafBaseDomain, p.partial[q].row.data(), cols);
        ok = verify_merkle_siblings(leaf, sel.at(q), rows, p.partial[q].path.siblings, root);
      }
    } else {
      ok = sel.all && p.n_rows == rows && p.n_cols == cols && p.encoded.size() == rows * cols &&
           build_row_tree<F>(kLeafBaseDomain, p.encoded, rows, cols).root() == root;
    }
    if (!ok) return false;
    payloads.push_back(std::move(p));
  }
  if (!r.empty()) return false;
  auto entry = [&](const Rows<F>& p, size_t q, size_t index, size_t col) {
    return p.all ? p.encoded[col * rows + index] : p.partial[q].row[col];
  };
  for (size_t q = 0; q < sel.size(); ++q) {
    size_t index = sel.at(q);
    for (size_t c = 0; c < cols; ++c) {
      F expected = F::zero();
      for (size_t b = 0; b < roots.size(); ++b) expected += weights[b] * entry(payloads[b], q, index, c);
      if (entry(payloads[roots.size()], q, index, c) != expected) return false;
    }
  }
  return true;
}

template <class F>
bool verify_batch(const PackedPcs<F>& pcs, const std::vector<Digest>& roots, const std::vector<F>& point, F claimed,
                  const uint8_t* bytes, size_t n, const std::vector<uint8_t>& ctx) {
  const int L = F::kLanes;
  const size_t lane_log = ilog2(L);
  const size_t blocks = roots.size();
  if (blocks < 2 || blocks > 128 || !is_pow2(blocks) || point.size() != pcs.log_n + ilog2(blocks) || n > 256u * 1024 * 1024)
    return false;
  const size_t split = ilog2(blocks);
  std::vector<F> outer(point.begin() + split, point.end() - lane_log);
  std::vector<F> low = equality_table(std::vector<F>(point.end() - lane_log, point.end()));
  std::vector<F> high = equality_table(std::vector<F>(point.begin(), point.begin() + split));
  ByteReader r(bytes, n);
  if (std::memcmp(r.take(8), "QAPKBAT1", 8) != 0 || r.field<F>() != claimed) return false;
  std::vector<F> evaluations(L);
  for (int i = 0; i < L; ++i) evaluations[i] = r.field<F>();
  if (projected_claim(evaluations, low) != claimed) return false;
  PackedTranscript<F> t = pcs.batch_transcript(roots, point, claimed, ctx);
  for (const F& v : evaluations) t.field(v);
  std::vector<F> powers = consecutive_powers(t.challenge(), L);
  F claim = F::zero();
  for (int i = 0; i < L; ++i) claim += powers[i] * evaluations[i];
  std::vector<F> positive, negative;
  for (size_t d = 1; d < blocks; ++d) positive.push_back(r.field<F>());
  for (size_t d = 1; d < blocks; ++d) negative.push_back(r.field<F>());
  t.bytes_str("block-packed-eo-cross");
  for (const F& v : positive) t.field(v);
  for (const F& v : negative) t.field(v);
  F ch = t.nonzero_challenge();
  {
    F inv = ch.inverse(), fwd = ch, bwd = inv;
    for (size_t i = 0; i < positive.size(); ++i) { claim += positive[i] * fwd + negative[i] * bwd; fwd *= ch; bwd *= inv; }
  }
  std::vector<F> fold_weights = consecutive_powers(ch.inverse(), blocks);
  std::vector<F> coefficients = folded_coefficients(high, powers, ch);
  Digest folded = r.digest();
  t.bytes(folded.data(), 32);
  std::vector<F> reduced;
  for (size_t k = 0; k < outer.size(); ++k) {
    F m[2] = {r.field<F>(), r.field<F>()};
    t.field(m[0]);
    t.field(m[1]);
    F c = t.challenge();
    claim = round_evaluation(claim, m, c);
    reduced.push_back(c);
  }
  F final_value = r.field<F>();
  if (claim != final_value * batch_weight(outer, reduced, coefficients)) return false;
  t.bytes_str("authenticated-codeword-fold-queries/v1");
  t.field(final_value);
  Digest seed = t.h.finalize();
  uint64_t blen = r.len();
  const uint8_t* bptr = r.take(blen);
  if (!verify_codeword_fold(*pcs.pp, roots, fold_weights, folded, seed, bptr, blen)) return false;
  uint64_t olen = r.len();
  const uint8_t* optr = r.take(olen);
  OpeningProof<F> op = opening_from_bytes<F>(optr, olen);
  uint64_t dlen = r.len();
  const uint8_t* dptr = r.take(dlen);
  DecideProof<F> dp = decide_from_bytes<F>(dptr, dlen);
  if (!r.empty()) return false;
  Reduction<F> red = verify_opening_reduction(*pcs.pp, folded, reduced, final_value, op);
  if (!red.ok) return false;
  return verify_decide(*pcs.pp, red, dp);
}

// ------------------------------------------------------------ single block
template <class F>
struct SingleBackend {
  virtual ~SingleBackend() {}
  virtual Digest commit() = 0;
  virtual std::vector<F> project(const std::vector<F>& outer) = 0;  // lanes; weights <- eq(outer)
  virtual void apply_images(const std::vector<F>& images) = 0;
  virtual void sumcheck_message(F m[2]) = 0;
  virtual void sumcheck_fold(F ch) = 0;
  virtual F sumcheck_final_value() = 0;
  virtual F sumcheck_final_weight() = 0;
  virtual const CodewordView<F>& codeword() = 0;
  virtual std::vector<F> opening(const std::vector<F>& point, size_t col_log, std::vector<F>& row_weights) = 0;
  virtual TopRoundAccel<F>* top_round_accel() { return nullptr; }
  virtual DecideAccel<F>* decide_accel() { return nullptr; }
};

// PackedPcs::open (packed.rs:294-393).
template <class F>
BatchOpening<F> open_single(const PackedPcs<F>& pcs, SingleBackend<F>& be, const Digest& root, const std::vector<F>& point,
                            const std::vector<uint8_t>& ctx) {
  const int L = F::kLanes;
  const size_t lane_log = ilog2(L);
  if (point.size() != pcs.log_n) fail(QF_E_INVALID_PARAMETERS, "packed opening profile or point mismatch");
  BatchOpening<F> out;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<F> outer(point.begin(), point.end() - lane_log);
  std::vector<F> lanes = be.project(outer);
  std::vector<F> low = equality_table(std::vector<F>(point.end() - lane_log, point.end()));
  F claimed = F::zero();
  for (int j = 0; j < L; ++j) claimed += lanes[j] * low[j];
  std::vector<F> evaluations = conjugates(lanes);
  if (projected_claim(evaluations, low) != claimed) fail(QF_E_INVALID_COMMITMENT, "projected claim");
  PackedTranscript<F> t = pcs.transcript(root, point, claimed, ctx);
  for (const F& v : evaluations) t.field(v);
  std::vector<F> powers = consecutive_powers(t.challenge(), L);
  F claim = F::zero();
  for (int i = 0; i < L; ++i) claim += powers[i] * evaluations[i];
  be.apply_images(weight_images(powers));
  out.times.projection_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  std::vector<std::array<F, 2>> rounds;
  std::vector<F> reduced;
  for (size_t k = 0; k < outer.size(); ++k) {
    F m[2];
    be.sumcheck_message(m);
    t.field(m[0]);
    t.field(m[1]);
    F c = t.challenge();
    claim = round_evaluation(claim, m, c);
    be.sumcheck_fold(c);
    rounds.push_back({m[0], m[1]});
    reduced.push_back(c);
  }
  F final_value = be.sumcheck_final_value();
  F final_weight = batch_weight(outer, reduced, powers);
  if (be.sumcheck_final_weight() != final_weight || claim != final_value * final_weight)
    fail(QF_E_INVALID_COMMITMENT, "sumcheck terminal");
  out.times.sumcheck_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  const CodewordView<F>& cw = be.codeword();
  const size_t col_log = ilog2(pcs.pp->extension_columns);
  std::vector<F> rw;
  std::vector<F> opening_vec = be.opening(reduced, col_log, rw);
  F actual = inner_product(opening_vec, tensor_weights(std::vector<F>(reduced.begin(), reduced.begin() + col_log)));
  OpenResult<F> op = open_with_reduction(*pcs.pp, cw, reduced, opening_vec, actual, rw, be.top_round_accel());
  if (op.claimed != final_value || !op.reduction.ok) fail(QF_E_INVALID_COMMITMENT, "native opening value");
  out.times.native_opening_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  DecideProof<F> dp = prove_decide(*pcs.pp, op.reduction, be.decide_accel());
  out.times.decide_ms = ms_since(t0);
  const std::vector<uint8_t> ob = opening_to_bytes(op.proof);
  const std::vector<uint8_t> db = decide_to_bytes(dp);
  ByteWriter w;
  w.bytes(F::kPackedMagic, 8);
  w.field(claimed);
  for (const F& v : evaluations) w.field(v);
  w.len(rounds.size());
  for (const auto& m : rounds) { w.field(m[0]); w.field(m[1]); }
  w.field(final_value);
  w.len(ob.size());
  w.bytes(ob.data(), ob.size());
  w.len(db.size());
  w.bytes(db.data(), db.size());
  out.claimed_value = claimed;
  out.wire = std::move(w.out);
  return out;
}

template <class F>
bool verify_single(const PackedPcs<F>& pcs, const Digest& root, const std::vector<F>& point, F claimed, const uint8_t* bytes,
                   size_t n, const std::vector<uint8_t>& ctx) {
  const int L = F::kLanes;
  const size_t lane_log = ilog2(L);
  if (point.size() != pcs.log_n || n > 256u * 1024 * 1024) return false;
  ByteReader r(bytes, n);
  if (std::memcmp(r.take(8), F::kPackedMagic, 8) != 0 || r.field<F>() != claimed) return false;
  std::vector<F> evaluations(L);
  for (int i = 0; i < L; ++i) evaluations[i] = r.field<F>();
  std::vector<F> low = equality_table(std::vector<F>(point.end() - lane_log, point.end()));
  if (projected_claim(evaluations, low) != claimed) return false;
  PackedTranscript<F> t = pcs.transcript(root, point, claimed, ctx);
  for (const F& v : evaluations) t.field(v);
  std::vector<F> powers = consecutive_powers(t.challenge(), L);
  F claim = F::zero();
  for (int i = 0; i < L; ++i) claim += powers[i] * evaluations[i];
  size_t count = r.len();
  if (count != pcs.log_n - lane_log) return false;
  std::vector<F> reduced;
  for (size_t k = 0; k < count; ++k) {
    F m[2] = {r.field<F>(), r.field<F>()};
    t.field(m[0]);
    t.field(m[1]);
    F c = t.challenge();
    claim = round_evaluation(claim, m, c);
    reduced.push_back(c);
  }
  F final_value = r.field<F>();
  std::vector<F> outer(point.begin(), point.end() - lane_log);
  if (claim != final_value * batch_weight(outer, reduced, powers)) return false;
  uint64_t olen = r.len();
  const uint8_t* optr = r.take(olen);
  OpeningProof<F> op = opening_from_bytes<F>(optr, olen);
  uint64_t dlen = r.len();
  const uint8_t* dptr = r.take(dlen);
  DecideProof<F> dp = decide_from_bytes<F>(dptr, dlen);
  if (!r.empty()) return false;
  Reduction<F> red = verify_opening_reduction(*pcs.pp, root, reduced, final_value, op);
  if (!red.ok) return false;
  return verify_decide(*pcs.pp, red, dp);
}

}  // namespace qf
