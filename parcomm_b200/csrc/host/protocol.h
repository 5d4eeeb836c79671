// Public-metadata ParComm over a packed QAFold PCS: BVA layout, compact
// tensor queries (TBV), the packed Laurent EO reduction, the outer BLAKE2s
// chaining transcript with serde_json-compatible absorption, and the
// bincode-fixint proof wire.
//
// Reference: qafold/f65521/src/layout.rs:34-155, tbv.rs:13-428,
// eo.rs:16-220, transcript.rs:8-70, field.rs:9-69, protocol.rs:18-327,
// main.rs:108-209 (demo inputs and benchmark points).
#pragma once
#include <array>
#include <cstdio>
#include <string>
#include <vector>

#include "packed.h"

namespace qf {

// ------------------------------------------------------------ layout
struct Shape { size_t rows, cols; };
struct Bucket { size_t matrix, row_offset, col_offset, rows, cols, physical_rows, physical_cols, offset; size_t len() const { return rows * cols; } };
struct Layout {
  std::vector<Shape> shapes;
  std::vector<Bucket> buckets;
  size_t active = 0, logical = 0;
};

inline std::vector<std::pair<size_t, size_t>> intervals(size_t length, size_t budget) {
  std::vector<size_t> sizes;
  size_t rem = length;
  while (rem > 0 && sizes.size() < budget) { size_t s = size_t(1) << ilog2(rem); sizes.push_back(s); rem -= s; }
  if (rem > 0) sizes.back() *= 2;
  std::vector<std::pair<size_t, size_t>> out;
  size_t off = 0;
  for (size_t s : sizes) { out.push_back({off, s}); off += s; }
  return out;
}

inline Layout make_layout(const std::vector<Shape>& shapes) {
  check(!shapes.empty() && shapes.size() <= 65536, "invalid matrix count");
  Layout L;
  L.shapes = shapes;
  for (size_t m = 0; m < shapes.size(); ++m) {
    const Shape& s = shapes[m];
    check(s.rows > 0 && s.cols > 0 && s.rows <= (size_t(1) << 30) && s.cols <= (size_t(1) << 30), "invalid matrix shape");
    for (auto [ro, r] : intervals(s.rows, 4))
      for (auto [co, c] : intervals(s.cols, 4)) {
        check(r * c <= (size_t(1) << 37), "matrix exceeds supported capacity");
        L.buckets.push_back({m, ro, co, r, c, std::min(r, s.rows - ro), std::min(c, s.cols - co), 0});
      }
  }
  std::stable_sort(L.buckets.begin(), L.buckets.end(), [](const Bucket& a, const Bucket& b) {
    if (a.len() != b.len()) return a.len() > b.len();
    if (a.matrix != b.matrix) return a.matrix < b.matrix;
    if (a.row_offset != b.row_offset) return a.row_offset < b.row_offset;
    return a.col_offset < b.col_offset;
  });
  size_t active = 0;
  for (Bucket& b : L.buckets) {
    b.offset = active;
    active += b.len();
    check(active <= (size_t(1) << 37), "collection exceeds supported capacity");
    check(b.offset % b.len() == 0, "unaligned BVA bucket");
  }
  L.active = active;
  L.logical = next_pow2(std::max<size_t>(active, 1024));
  return L;
}

// Dense row-major matrices -> BVA vector of `active` entries.
template <class T>
std::vector<T> layout_encode(const Layout& L, const std::vector<std::vector<T>>& matrices) {
  check(matrices.size() == L.shapes.size(), "matrix count mismatch");
  for (size_t i = 0; i < matrices.size(); ++i) check(matrices[i].size() == L.shapes[i].rows * L.shapes[i].cols, "matrix length mismatch");
  std::vector<T> v(L.active, T(0));
  for (const Bucket& b : L.buckets)
    for (size_t r = 0; r < b.physical_rows; ++r) {
      size_t src = (b.row_offset + r) * L.shapes[b.matrix].cols + b.col_offset;
      size_t dst = b.offset + r * b.cols;
      std::memcpy(&v[dst], &matrices[b.matrix][src], b.physical_cols * sizeof(T));
    }
  return v;
}
template <class T>
void validate_values(const Layout& L, const T* v, size_t n) {
  check(n == L.active, "active BVA length mismatch");
  for (const Bucket& b : L.buckets)
    for (size_t r = 0; r < b.rows; ++r) {
      size_t valid = r < b.physical_rows ? b.physical_cols : 0;
      for (size_t i = b.offset + r * b.cols + valid; i < b.offset + (r + 1) * b.cols; ++i)
        check(v[i] == 0, "nonzero boundary padding");
    }
}

// ------------------------------------------------------------ JSON (serde_json compact)
struct Json {
  std::string s;
  void raw(const char* x) { s += x; }
  void num(uint64_t v) { s += std::to_string(v); }
  // serde_json's byte arrays: "[b0,b1,...]" in decimal.  The digits of each
  // byte value come from a table (a large collection's claims hold about
  // 10^5 bytes).
  void bytes(const uint8_t* p, size_t n) {
    static const std::array<std::array<char, 4>, 256> digits = [] {
      std::array<std::array<char, 4>, 256> t{};
      for (int v = 0; v < 256; ++v) {
        const std::string d = std::to_string(v);
        t[v][0] = char(d.size());
        std::memcpy(&t[v][1], d.data(), d.size());
      }
      return t;
    }();
    s += '[';
    for (size_t i = 0; i < n; ++i) {
      if (i) s += ',';
      s.append(&digits[p[i]][1], size_t(digits[p[i]][0]));
    }
    s += ']';
  }
  template <class F> void scalar(const F& v) { uint8_t e[F::kBytes]; v.to_bytes(e); bytes(e, F::kBytes); }
  template <class F> void scalars(const std::vector<F>& vs) {
    s += '[';
    for (size_t i = 0; i < vs.size(); ++i) { if (i) s += ','; scalar(vs[i]); }
    s += ']';
  }
};

struct Config { size_t chunk_log = 30, packed_log = 4, query_rf_bits = 100; };
struct Commitment {
  uint32_t version = 2;
  Config config;
  std::vector<Shape> shapes;
  Digest parameter_digest{};
  std::vector<Digest> roots;
};
inline std::string commitment_json(const Commitment& c) {
  Json j;
  j.raw("{\"version\":"); j.num(c.version);
  j.raw(",\"config\":{\"chunk_log\":"); j.num(c.config.chunk_log);
  j.raw(",\"packed_log\":"); j.num(c.config.packed_log);
  j.raw(",\"query_rf_bits\":"); j.num(c.config.query_rf_bits);
  j.raw("},\"shapes\":[");
  for (size_t i = 0; i < c.shapes.size(); ++i) {
    if (i) j.raw(",");
    j.raw("{\"rows\":"); j.num(c.shapes[i].rows); j.raw(",\"cols\":"); j.num(c.shapes[i].cols); j.raw("}");
  }
  j.raw("],\"parameter_digest\":"); j.bytes(c.parameter_digest.data(), 32);
  j.raw(",\"roots\":[");
  for (size_t i = 0; i < c.roots.size(); ++i) { if (i) j.raw(","); j.bytes(c.roots[i].data(), 32); }
  j.raw("]}");
  return j.s;
}

template <class F>
struct Claim {
  std::vector<F> row, col;
  F value;
};
template <class F>
std::string claims_json(const std::vector<Claim<F>>& claims) {
  Json j;
  size_t coords = 0;
  for (const auto& c : claims) coords += c.row.size() + c.col.size() + 1;
  j.s.reserve(coords * (F::kBytes * 4 + 2) + claims.size() * 32 + 2);
  j.raw("[");
  for (size_t i = 0; i < claims.size(); ++i) {
    if (i) j.raw(",");
    j.raw("{\"row\":"); j.scalars(claims[i].row);
    j.raw(",\"col\":"); j.scalars(claims[i].col);
    j.raw(",\"value\":"); j.scalar(claims[i].value);
    j.raw("}");
  }
  j.raw("]");
  return j.s;
}

// ------------------------------------------------------------ outer transcript
template <class F>
struct Transcript {
  Digest state;
  uint64_t counter = 0;
  Transcript() { const char* d = F::kPublicDomain; state = blake2s(d, std::strlen(d)); }
  void bytes(const char* label, const void* b, size_t n) {
    Blake2s h;
    h.update(state);
    size_t ll = std::strlen(label);
    h.update_u64(ll);
    h.update(label, ll);
    h.update_u64(n);
    h.update(b, n);
    state = h.finalize();
  }
  void object(const char* label, const std::string& json) { bytes(label, json.data(), json.size()); }
  void scalar(const char* label, const F& v) { uint8_t e[F::kBytes]; v.to_bytes(e); bytes(label, e, F::kBytes); }
  F challenge(const char* label) {
    for (;;) {
      uint64_t c = counter++;
      auto b = le64(c);
      bytes(label, b.data(), 8);
      F v;
      if (F::from_uniform_bytes(state.data(), v)) return v;
    }
  }
  F nonzero(const char* label) { for (;;) { F v = challenge(label); if (!v.is_zero()) return v; } }
  F fold_challenge(size_t packed_log) {
    for (;;) {
      F v = nonzero("eo-fold");
      F p = v;
      bool ok = true;
      F minus_one = -F::one();
      for (size_t i = 0; i < std::max<size_t>(packed_log, 1); ++i) { ok = ok && p != minus_one; p = p * p; }
      if (ok) return v;
    }
  }
};

// ------------------------------------------------------------ TBV
template <class F>
F monomial_weight(size_t index, const F* point_low, size_t n) {
  F w = F::one();
  for (size_t bit = 0; bit < n; ++bit)
    if ((index >> bit) & 1) w = w * point_low[bit];
  return w;
}
template <class F>
F equality_weight(size_t index, const std::vector<F>& msb) {
  F w = F::one();
  for (size_t c = 0; c < msb.size(); ++c) w = w * (((index >> (msb.size() - 1 - c)) & 1) ? msb[c] : F::one() - msb[c]);
  return w;
}

template <class F>
struct Term {
  size_t offset;
  F scale;
  std::vector<std::array<F, 2>> factors;  // low-bit first
  size_t len() const { return size_t(1) << factors.size(); }
  F weight(size_t index) const {
    F v = scale;
    for (size_t b = 0; b < factors.size(); ++b) v = v * factors[b][(index >> b) & 1];
    return v;
  }
  F evaluation(const std::vector<F>& point_low) const {
    F local = scale;
    for (size_t k = 0; k < factors.size(); ++k) local = local * (factors[k][0] + factors[k][1] * point_low[k]);
    return local * monomial_weight(offset >> factors.size(), point_low.data() + factors.size(), point_low.size() - factors.size());
  }
};
// Tensor weights of LSB-first factor pairs (tbv.rs:45-76).
template <class F>
std::vector<F> factor_weights(const std::array<F, 2>* factors, size_t n) {
  std::vector<F> r(1, F::one());
  for (size_t k = 0; k < n; ++k) {
    size_t len = r.size();
    r.resize(2 * len);
#pragma omp parallel for if (len >= 4096)
    for (long i = 0; i < long(len); ++i) { r[len + i] = r[i] * factors[k][1]; r[i] = r[i] * factors[k][0]; }
  }
  return r;
}
template <class F>
struct Query {
  std::vector<Term<F>> terms;
  F claim;
  F evaluation(const std::vector<F>& point_low) const {
    F s = F::zero();
    for (const auto& t : terms) s += t.evaluation(point_low);
    return s;
  }
};

inline std::vector<std::pair<size_t, size_t>> aligned_intervals(size_t start, size_t end) {
  std::vector<std::pair<size_t, size_t>> out;
  while (start < end) {
    size_t fit = ilog2(end - start);
    size_t bits = start == 0 ? fit : std::min<size_t>(fit, __builtin_ctzll(start));
    size_t len = size_t(1) << bits;
    out.push_back({start, len});
    start += len;
  }
  return out;
}
template <class F>
Term<F> compact_term(Term<F> t) {
  while (!t.factors.empty()) {
    auto pair = t.factors.back();
    size_t fixed;
    if (pair[0].is_zero()) fixed = 1;
    else if (pair[1].is_zero()) fixed = 0;
    else break;
    size_t bit = t.factors.size() - 1;
    t.scale = t.scale * pair[fixed];
    t.offset += fixed << bit;
    t.factors.pop_back();
  }
  return t;
}
template <class F>
void validate_claims(const Layout& L, const std::vector<Claim<F>>& claims) {
  check(claims.size() == L.shapes.size(), "claim count mismatch");
  for (size_t i = 0; i < claims.size(); ++i)
    check(claims[i].row.size() == size_t(ilog2(next_pow2(L.shapes[i].rows))) &&
              claims[i].col.size() == size_t(ilog2(next_pow2(L.shapes[i].cols))),
          "point dimension mismatch");
}

template <class F>
Query<F> compile(const Layout& L, const std::vector<Claim<F>>& claims, Transcript<F>& t) {
  validate_claims(L, claims);
  std::vector<F> batch_point;
  for (int i = 0; i < ilog2(next_pow2(claims.size())); ++i) batch_point.push_back(t.challenge("batch"));
  std::vector<F> coeff;
  for (size_t i = 0; i < claims.size(); ++i) coeff.push_back(equality_weight(i, batch_point));
  Query<F> q;
  q.claim = F::zero();
  for (size_t i = 0; i < claims.size(); ++i) q.claim += coeff[i] * claims[i].value;
  for (const Bucket& b : L.buckets) {
    const auto& row = claims[b.matrix].row;
    const auto& col = claims[b.matrix].col;
    F scale = coeff[b.matrix] * monomial_weight(b.row_offset, row.data(), row.size()) * monomial_weight(b.col_offset, col.data(), col.size());
    Term<F> term{b.offset, scale, {}};
    for (int k = 0; k < ilog2(b.cols); ++k) term.factors.push_back({F::one(), col[k]});
    for (int k = 0; k < ilog2(b.rows); ++k) term.factors.push_back({F::one(), row[k]});
    q.terms.push_back(std::move(term));
  }
  std::vector<F> pp;
  for (int i = 0; i < ilog2(L.logical); ++i) pp.push_back(t.challenge("padding-point"));
  F mixing = t.nonzero("padding-mix");
  for (const Bucket& b : L.buckets) {
    size_t col_bits = ilog2(b.cols), bits = ilog2(b.len());
    std::vector<std::array<size_t, 4>> rects;
    for (auto [s, l] : aligned_intervals(b.physical_rows, b.rows)) rects.push_back({s, l, 0, b.cols});
    for (auto [rs, rl] : aligned_intervals(0, b.physical_rows))
      for (auto [cs, cl] : aligned_intervals(b.physical_cols, b.cols)) rects.push_back({rs, rl, cs, cl});
    for (auto [rs, rl, cs, cl] : rects) {
      std::vector<std::array<F, 2>> factors;
      for (size_t k = 0; k < bits; ++k) factors.push_back({F::one(), pp[k]});
      for (size_t bit = ilog2(cl); bit < col_bits; ++bit) factors[bit][1 - ((cs >> bit) & 1)] = F::zero();
      for (size_t bit = ilog2(rl); bit < size_t(ilog2(b.rows)); ++bit) factors[col_bits + bit][1 - ((rs >> bit) & 1)] = F::zero();
      Term<F> term{b.offset, mixing * monomial_weight(b.offset >> bits, pp.data() + bits, pp.size() - bits), std::move(factors)};
      q.terms.push_back(compact_term(std::move(term)));
    }
  }
  for (auto [off, len] : aligned_intervals(L.active, L.logical)) {
    size_t bits = ilog2(len);
    Term<F> term{off, mixing * monomial_weight(off >> bits, pp.data() + bits, pp.size() - bits), {}};
    for (size_t k = 0; k < bits; ++k) term.factors.push_back({F::one(), pp[k]});
    q.terms.push_back(std::move(term));
  }
  return q;
}

// ------------------------------------------------------------ EO
template <class F>
struct EoProof {
  std::vector<F> positive, negative;
  std::vector<std::array<F, 2>> rounds;
  F value, query;
};
template <class F>
struct Terminal {
  F value, scale;
  std::vector<F> point_msb;
};

// Heavy EO steps over the resident BVA (cross terms, packed witness and query
// fold, binary rounds).
template <class F>
struct EoBackend {
  virtual ~EoBackend() {}
  virtual void cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) = 0;
  // Builds witness[logical/stride] and folded query; returns their dot product.
  virtual F eo_build(const Query<F>& q, F challenge, F inverse, size_t logical, size_t stride) = 0;
  virtual std::array<F, 2> eo_round_cross() = 0;
  virtual void eo_round_fold(F inv, F ch) = 0;
  virtual std::array<F, 2> eo_terminal() = 0;  // witness[0], query[0]
};

template <class F>
std::string scalars_json(const std::vector<F>& v) { Json j; j.scalars(v); return j.s; }

template <class F>
F eo_update_claim(F claim, const std::vector<F>& pos, const std::vector<F>& neg, F ch) {
  F inv = ch.inverse(), fwd = ch, bwd = inv;
  for (size_t i = 0; i < pos.size(); ++i) { claim += pos[i] * fwd + neg[i] * bwd; fwd *= ch; bwd *= inv; }
  return claim;
}
template <class F>
Terminal<F> eo_normalized(const std::vector<F>& challenges, F value) {
  Terminal<F> t;
  t.scale = F::one();
  for (const F& c : challenges) {
    F mono = c.inverse();
    F factor = F::one() + mono;
    t.point_msb.push_back(mono * factor.inverse());
    t.scale *= factor;
  }
  std::reverse(t.point_msb.begin(), t.point_msb.end());
  t.value = value;
  return t;
}

template <class F>
std::pair<EoProof<F>, Terminal<F>> eo_prove(EoBackend<F>& be, size_t logical, size_t stride, const Query<F>& q, Transcript<F>& t) {
  EoProof<F> proof;
  be.cross_terms(q, stride, proof.positive, proof.negative);
  t.object("packed-positive", scalars_json(proof.positive));
  t.object("packed-negative", scalars_json(proof.negative));
  F ch = t.fold_challenge(ilog2(stride));
  std::vector<F> challenges;
  F p = ch;
  for (int i = 0; i < ilog2(stride); ++i) { challenges.push_back(p); p = p * p; }
  F inv = ch.inverse();
  F dot = be.eo_build(q, ch, inv, logical, stride);
  F claim = eo_update_claim(q.claim, proof.positive, proof.negative, ch);
  check(dot == claim, "packed reduction claim mismatch");
  for (size_t len = logical / stride; len > 1; len /= 2) {
    std::array<F, 2> cross = be.eo_round_cross();
    Json j;
    j.raw("[");
    j.scalar(cross[0]);
    j.raw(",");
    j.scalar(cross[1]);
    j.raw("]");
    t.object("binary-cross", j.s);
    F c = t.fold_challenge(1);
    F ci = c.inverse();
    claim += cross[0] * c + cross[1] * ci;
    challenges.push_back(c);
    be.eo_round_fold(ci, c);
    proof.rounds.push_back(cross);
  }
  std::array<F, 2> term = be.eo_terminal();
  check(claim == term[0] * term[1] && q.evaluation(challenges) == term[1], "EO terminal mismatch");
  t.scalar("terminal-value", term[0]);
  t.scalar("terminal-query", term[1]);
  proof.value = term[0];
  proof.query = term[1];
  return {proof, eo_normalized(challenges, term[0])};
}

template <class F>
Terminal<F> eo_verify(const EoProof<F>& proof, size_t logical, size_t stride, const Query<F>& q, Transcript<F>& t) {
  check(proof.positive.size() == stride - 1 && proof.negative.size() == stride - 1 &&
            proof.rounds.size() == size_t(ilog2(logical / stride)),
        "EO proof dimensions");
  t.object("packed-positive", scalars_json(proof.positive));
  t.object("packed-negative", scalars_json(proof.negative));
  F ch = t.fold_challenge(ilog2(stride));
  F claim = eo_update_claim(q.claim, proof.positive, proof.negative, ch);
  std::vector<F> challenges;
  F p = ch;
  for (int i = 0; i < ilog2(stride); ++i) { challenges.push_back(p); p = p * p; }
  for (const auto& r : proof.rounds) {
    Json j;
    j.raw("[");
    j.scalar(r[0]);
    j.raw(",");
    j.scalar(r[1]);
    j.raw("]");
    t.object("binary-cross", j.s);
    F c = t.fold_challenge(1);
    claim += r[0] * c + r[1] * c.inverse();
    challenges.push_back(c);
  }
  check(claim == proof.value * proof.query, "EO scalar relation rejected");
  check(q.evaluation(challenges) == proof.query, "TBV terminal evaluation rejected");
  t.scalar("terminal-value", proof.value);
  t.scalar("terminal-query", proof.query);
  return eo_normalized(challenges, proof.value);
}

// ------------------------------------------------------------ proof wire (bincode fixint)
template <class F>
struct Proof {
  EoProof<F> eo;
  F opening_value;
  std::vector<uint8_t> opening_proof;
};
template <class F>
std::vector<uint8_t> proof_to_bytes(const Proof<F>& p) {
  ByteWriter w;
  w.out.reserve(64 + (p.eo.positive.size() + p.eo.negative.size() + 2 * p.eo.rounds.size() + 3) * F::kBytes +
                p.opening_proof.size());
  w.len(p.eo.positive.size());
  for (const F& v : p.eo.positive) w.field(v);
  w.len(p.eo.negative.size());
  for (const F& v : p.eo.negative) w.field(v);
  w.len(p.eo.rounds.size());
  for (const auto& r : p.eo.rounds) { w.field(r[0]); w.field(r[1]); }
  w.field(p.eo.value);
  w.field(p.eo.query);
  w.len(1);
  w.field(p.opening_value);
  w.len(p.opening_proof.size());
  w.bytes(p.opening_proof.data(), p.opening_proof.size());
  return std::move(w.out);
}
template <class F>
Proof<F> proof_from_bytes(const uint8_t* d, size_t n) {
  check(n <= 256u * 1024 * 1024, "oversize ParComm proof");
  ByteReader r(d, n);
  Proof<F> p;
  auto vec = [&](std::vector<F>& out) {
    uint64_t k = r.len();
    if (k > r.remaining() / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "vector length");
    for (uint64_t i = 0; i < k; ++i) out.push_back(r.field<F>());
  };
  vec(p.eo.positive);
  vec(p.eo.negative);
  uint64_t nr = r.len();
  if (nr > r.remaining() / (2 * F::kBytes)) fail(QF_E_INVALID_COMMITMENT, "rounds length");
  for (uint64_t i = 0; i < nr; ++i) { F a = r.field<F>(); F b = r.field<F>(); p.eo.rounds.push_back({a, b}); }
  p.eo.value = r.field<F>();
  p.eo.query = r.field<F>();
  uint64_t no = r.len();
  check(no == 1, "PCS opening count");
  p.opening_value = r.field<F>();
  uint64_t pl = r.len();
  const uint8_t* pp = r.take(pl);
  p.opening_proof.assign(pp, pp + pl);
  if (!r.empty()) fail(QF_E_INVALID_COMMITMENT, "trailing proof bytes");
  return p;
}

template <class F>
std::vector<uint8_t> opening_context(const Digest& state, size_t block) {
  const char* d = F::kTerminalDomain;
  std::vector<uint8_t> b(d, d + std::strlen(d));
  b.insert(b.end(), state.begin(), state.end());
  auto bl = le64(block);
  b.insert(b.end(), bl.begin(), bl.end());
  return b;
}

// ------------------------------------------------------------ parameters
template <class F>
struct Parameters {
  Layout layout;
  Config config;
  PackedPcs<F> pcs;
  size_t block_len = 0;
  size_t blocks() const { return layout.logical / block_len; }
  size_t chunk_log() const { return ilog2(block_len); }
};

template <class F>
std::unique_ptr<Parameters<F>> make_parameters(const std::vector<Shape>& shapes, const Config& config,
                                               SetupAccel<F>* accel = nullptr) {
  check(config.chunk_log >= 10 && config.chunk_log <= 30 && config.packed_log >= 1 && config.packed_log <= 6 &&
            config.query_rf_bits >= 32 && config.query_rf_bits <= 120,
        "invalid ParComm config");
  auto p = std::make_unique<Parameters<F>>();
  p->layout = make_layout(shapes);
  p->config = config;
  size_t chunk_log = std::min<size_t>(config.chunk_log, ilog2(p->layout.logical));
  p->block_len = size_t(1) << chunk_log;
  check(p->layout.logical / p->block_len <= 128, "at most 128 PCS blocks are supported");
  std::array<uint8_t, 32> seed;
  seed.fill(0x51);
  p->pcs = PackedPcs<F>::create(chunk_log, 32, config.query_rf_bits, seed, accel);
  return p;
}

template <class F>
Commitment make_statement(const Parameters<F>& P, const std::vector<Digest>& roots) {
  Commitment c;
  c.config = P.config;
  c.shapes = P.layout.shapes;
  c.parameter_digest = P.pcs.parameter_digest();
  c.roots = roots;
  return c;
}

template <class F>
Transcript<F> statement_transcript(const Parameters<F>& P, const Commitment& st, const std::vector<Claim<F>>& claims) {
  check(st.version == 2 && st.config.chunk_log == P.config.chunk_log && st.config.packed_log == P.config.packed_log &&
            st.config.query_rf_bits == P.config.query_rf_bits && st.shapes.size() == P.layout.shapes.size() &&
            st.parameter_digest == P.pcs.parameter_digest() && st.roots.size() == P.blocks(),
        "commitment/parameter mismatch");
  for (size_t i = 0; i < st.shapes.size(); ++i)
    check(st.shapes[i].rows == P.layout.shapes[i].rows && st.shapes[i].cols == P.layout.shapes[i].cols,
          "commitment/parameter mismatch");
  validate_claims(P.layout, claims);
  Transcript<F> t;
  t.object("collection", commitment_json(st));
  t.object("claims", claims_json(claims));
  return t;
}

// Witness-free verifier (protocol.rs:266-320).
template <class F>
bool verify_proof(const Parameters<F>& P, const Commitment& st, const std::vector<Claim<F>>& claims, const Proof<F>& proof) {
  Transcript<F> t = statement_transcript(P, st, claims);
  Query<F> q = compile(P.layout, claims, t);
  Terminal<F> term = eo_verify(proof.eo, P.layout.logical, size_t(1) << P.config.packed_log, q, t);
  std::vector<uint8_t> ctx = opening_context<F>(t.state, 0);
  bool ok;
  if (st.roots.size() > 1)
    ok = verify_batch(P.pcs, st.roots, term.point_msb, proof.opening_value, proof.opening_proof.data(), proof.opening_proof.size(), ctx);
  else
    ok = verify_single(P.pcs, st.roots[0], term.point_msb, proof.opening_value, proof.opening_proof.data(), proof.opening_proof.size(), ctx);
  if (!ok) fail(QF_E_INVALID_COMMITMENT, "PCS opening rejected");
  check(proof.opening_value * term.scale == term.value, "PCS terminal aggregate rejected");
  return true;
}

// Benchmark points (main.rs:190-204): derived from the committed statement.
template <class F>
std::vector<std::pair<std::vector<F>, std::vector<F>>> benchmark_points(const Commitment& st) {
  Transcript<F> t;
  t.object("benchmark-points", commitment_json(st));
  std::vector<std::pair<std::vector<F>, std::vector<F>>> pts;
  for (const Shape& s : st.shapes) {
    std::vector<F> r, c;
    for (int i = 0; i < ilog2(next_pow2(s.rows)); ++i) r.push_back(t.challenge("row"));
    for (int i = 0; i < ilog2(next_pow2(s.cols)); ++i) c.push_back(t.challenge("col"));
    pts.push_back({r, c});
  }
  return pts;
}

}  // namespace qf
