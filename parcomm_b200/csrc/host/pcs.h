// The QAFold polynomial commitment over a full extension field: parameters,
// setup commitments, recursive opening, its verifier, and the canonical wire.
//
// Reference: ShortQaFoldPC (qafold_short_pc.rs:326-905), round provers and
// verifiers (1022-1790), LiteBullet (1895-1999), parameter digest
// (2271-2325), extension commits (2327-2362), projections and folds
// (2641-2760), wire codecs (240-320, 3104-3420); direct-interleaved setup
// commitments (qafold_short_setup.rs:203-243, 427-536, 655-897).
#pragma once
#include <memory>
#include <optional>
#include <vector>

#include "chacha.h"
#include "field65521.h"
#include "fieldkb.h"
#include "merkle.h"
#include "qacode.h"
#include "sections.h"

namespace qf {

// ------------------------------------------------------------ small helpers
template <class F>
F inner_product(const std::vector<F>& a, const std::vector<F>& b) {
  if (a.size() != b.size()) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "inner product length");
  F s = F::zero();
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
template <class F>
F tensor_weight_at(const std::vector<F>& point, size_t pos) {
  F r = F::one();
  for (size_t bit = 0; bit < point.size(); ++bit)
    if ((pos >> bit) & 1) r *= point[point.size() - bit - 1];
  return r;
}
template <class F>
std::vector<F> tensor_weights_prefix(const std::vector<F>& point, size_t prefix_len) {
  if (point.size() >= 64) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "prefix point");
  size_t full = size_t(1) << point.size();
  if (prefix_len == 0 || prefix_len > full) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "prefix length");
  std::vector<F> out(prefix_len);
  for (size_t i = 0; i < prefix_len; ++i) out[i] = tensor_weight_at(point, i);
  return out;
}
template <class F>
F tensor_inner_product(const std::vector<F>& l, const std::vector<F>& r) {
  if (l.size() != r.size()) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "tensor inner product");
  F p = F::one();
  for (size_t i = 0; i < l.size(); ++i) p = p * (F::one() + l[i] * r[i]);
  return p;
}
template <class F>
bool mle_eval(const std::vector<F>& values, const std::vector<F>& point, F& out) {
  if (values.empty() || point.size() >= 64 || values.size() != (size_t(1) << point.size())) return false;
  std::vector<F> f = values;
  size_t len = f.size();
  for (const F& ch : point) {
    size_t half = len / 2;
    for (size_t i = 0; i < half; ++i) f[i] += f[i + half] * ch;
    len = half;
  }
  out = f[0];
  return true;
}

// ------------------------------------------------------------ proof structs
struct Path { std::vector<Digest> siblings; };
template <class F>
struct RowQuery {
  std::vector<F> row;
  Path path;
};
// Partial sampled rows, or a complete column-major codeword.
template <class F>
struct Rows {
  bool all = false;
  std::vector<RowQuery<F>> partial;
  std::vector<F> encoded;
  size_t n_rows = 0, n_cols = 0;
  size_t query_count() const { return all ? n_rows : partial.size(); }
};
template <class F>
struct ExtRound {
  Digest root{};
  Rows<F> rows;
};
template <class F>
struct OpeningProof {
  std::vector<F> responses;
  Rows<F> top;
  std::vector<ExtRound<F>> ext_rounds;
  std::vector<F> base_vector;
};
template <class F>
struct PendingH {
  size_t level;
  F value;
  std::vector<F> left_point, right_point;
  bool operator==(const PendingH& o) const {
    return level == o.level && value == o.value && left_point == o.left_point && right_point == o.right_point;
  }
};
template <class F>
struct Reduction {
  bool ok = false;
  std::vector<PendingH<F>> pending;
};

// ------------------------------------------------------------ wire helpers
struct ByteWriter {
  std::vector<uint8_t> out;
  void bytes(const void* p, size_t n) { const uint8_t* b = (const uint8_t*)p; out.insert(out.end(), b, b + n); }
  void u8(uint8_t v) { out.push_back(v); }
  void len(uint64_t v) { put_u64(out, v); }
  void digest(const Digest& d) { bytes(d.data(), 32); }
  template <class F> void field(const F& v) { uint8_t e[F::kBytes]; v.to_bytes(e); bytes(e, F::kBytes); }
};
struct ByteReader {
  const uint8_t* p;
  size_t n, cur = 0;
  ByteReader(const uint8_t* d, size_t len) : p(d), n(len) {}
  size_t remaining() const { return n - cur; }
  bool empty() const { return cur == n; }
  const uint8_t* take(size_t k) {
    if (k > n - cur) fail(QF_E_INVALID_COMMITMENT, "truncated proof");
    const uint8_t* r = p + cur;
    cur += k;
    return r;
  }
  uint8_t u8() { return *take(1); }
  uint64_t len() { const uint8_t* b = take(8); uint64_t v = 0; for (int i = 0; i < 8; ++i) v |= uint64_t(b[i]) << (8 * i); return v; }
  Digest digest() { Digest d; std::memcpy(d.data(), take(32), 32); return d; }
  template <class F> F field() {
    F v;
    if (!F::from_bytes(take(F::kBytes), v)) fail(QF_E_INVALID_COMMITMENT, "non-canonical field element");
    return v;
  }
};

template <class F>
void write_path(ByteWriter& w, const Path& p) {
  w.len(p.siblings.size());
  for (const Digest& d : p.siblings) w.digest(d);
}
template <class F>
void write_rows(ByteWriter& w, const Rows<F>& r) {
  if (!r.all) {
    w.u8(0);
    w.len(r.partial.size());
    for (const auto& q : r.partial) {
      w.len(q.row.size());
      for (const F& v : q.row) w.field(v);
      write_path<F>(w, q.path);
    }
  } else {
    w.u8(1);
    w.len(r.n_rows);
    w.len(r.n_cols);
    w.len(r.encoded.size());
    for (const F& v : r.encoded) w.field(v);
  }
}
inline Path read_path(ByteReader& r) {
  uint64_t n = r.len();
  if (n > r.remaining() / 32) fail(QF_E_INVALID_COMMITMENT, "path length");
  Path p;
  for (uint64_t i = 0; i < n; ++i) p.siblings.push_back(r.digest());
  return p;
}
template <class F>
Rows<F> read_rows(ByteReader& r) {
  Rows<F> rows;
  uint8_t mode = r.u8();
  if (mode == 0) {
    uint64_t n = r.len();
    if (n > r.remaining() / 16) fail(QF_E_INVALID_COMMITMENT, "row count");
    for (uint64_t i = 0; i < n; ++i) {
      RowQuery<F> q;
      uint64_t len = r.len();
      if (r.remaining() < 8 || len > (r.remaining() - 8) / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "row length");
      for (uint64_t j = 0; j < len; ++j) q.row.push_back(r.field<F>());
      q.path = read_path(r);
      rows.partial.push_back(std::move(q));
    }
  } else if (mode == 1) {
    rows.all = true;
    rows.n_rows = r.len();
    rows.n_cols = r.len();
    uint64_t len = r.len();
    unsigned __int128 prod = (unsigned __int128)rows.n_rows * rows.n_cols;
    if (prod != len || len > r.remaining() / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "all-rows length");
    rows.encoded.reserve(len);
    for (uint64_t j = 0; j < len; ++j) rows.encoded.push_back(r.field<F>());
  } else {
    fail(QF_E_INVALID_COMMITMENT, "row mode");
  }
  return rows;
}

template <class F>
std::vector<uint8_t> opening_to_bytes(const OpeningProof<F>& p) {
  ByteWriter w;
  w.bytes("QFSHORT2", 8);
  w.len(p.responses.size());
  for (const F& v : p.responses) w.field(v);
  write_rows(w, p.top);
  w.len(p.ext_rounds.size());
  for (const auto& r : p.ext_rounds) { w.digest(r.root); write_rows(w, r.rows); }
  w.len(p.base_vector.size());
  for (const F& v : p.base_vector) w.field(v);
  return std::move(w.out);
}
template <class F>
OpeningProof<F> opening_from_bytes(const uint8_t* d, size_t n) {
  ByteReader r(d, n);
  if (std::memcmp(r.take(8), "QFSHORT2", 8) != 0) fail(QF_E_INVALID_COMMITMENT, "opening magic");
  OpeningProof<F> p;
  uint64_t nr = r.len();
  if (nr > r.remaining() / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "responses length");
  for (uint64_t i = 0; i < nr; ++i) p.responses.push_back(r.field<F>());
  p.top = read_rows<F>(r);
  uint64_t ne = r.len();
  if (ne > (r.remaining() >= 8 ? r.remaining() - 8 : 0) / 33) fail(QF_E_INVALID_COMMITMENT, "rounds length");
  for (uint64_t i = 0; i < ne; ++i) {
    ExtRound<F> er;
    er.root = r.digest();
    er.rows = read_rows<F>(r);
    p.ext_rounds.push_back(std::move(er));
  }
  uint64_t nb = r.len();
  if (nb > r.remaining() / F::kBytes) fail(QF_E_INVALID_COMMITMENT, "base vector length");
  for (uint64_t i = 0; i < nb; ++i) p.base_vector.push_back(r.field<F>());
  if (!r.empty()) fail(QF_E_INVALID_COMMITMENT, "trailing opening bytes");
  return p;
}

// ------------------------------------------------------------ parameters
struct SetupShape {
  size_t level = 0, encoded_rows = 0, message_rows = 0, t_cols = 0, t_elements = 0, t_last_len = 0, h_cols = 0;
  bool operator==(const SetupShape& o) const {
    return level == o.level && encoded_rows == o.encoded_rows && message_rows == o.message_rows && t_cols == o.t_cols &&
           t_elements == o.t_elements && t_last_len == o.t_last_len && h_cols == o.h_cols;
  }
  size_t total_cols() const { return t_cols + h_cols; }
  void validate() const {
    if (level == 0 || !is_pow2(encoded_rows) || !is_pow2(message_rows) || encoded_rows < message_rows ||
        encoded_rows % message_rows || !is_pow2(h_cols))
      fail(QF_E_ENCODING, "setup shape");
    if (t_cols == 0 && (t_elements || t_last_len)) fail(QF_E_ENCODING, "setup shape t");
  }
};

template <class F>
struct SetupLevel {
  Digest root{};
  SetupShape shape;
  std::vector<F> encoded;  // column-major, encoded_rows x h_cols
  MerkleTree tree;
};

template <class F>
void absorb_field_metadata(Blake2s& h) {
  absorb_framed(h, "field-name", F::kName, std::strlen(F::kName));
  absorb_framed_u64(h, "modulus", F::modulus_u64());
  absorb_framed_u64(h, "canonical-bytes", F::kBytes);
  absorb_framed_u64(h, "extension-degree", 1);
}
inline void absorb_setup_shape(Blake2s& h, const SetupShape& s) {
  absorb_framed_u64(h, "level", s.level);
  absorb_framed_u64(h, "encoded-rows", s.encoded_rows);
  absorb_framed_u64(h, "message-rows", s.message_rows);
  absorb_framed_u64(h, "t-columns", s.t_cols);
  absorb_framed_u64(h, "t-elements", s.t_elements);
  absorb_framed_u64(h, "t-last-length", s.t_last_len);
  absorb_framed_u64(h, "h-columns", s.h_cols);
}
// The bytes a setup row's leaf hash absorbs before its framed row index:
// the domain, the field metadata (absorb_field_metadata), the setup mode and
// the shape (absorb_setup_shape), framed.
template <class F>
std::vector<uint8_t> setup_row_prefix(const SetupShape& s) {
  std::vector<uint8_t> b;
  auto u64 = [&](const char* label, uint64_t v) {
    const auto w = le64(v);
    append_frame(b, label, w.data(), 8);
  };
  const char* dom = "qafold-short/setup-base-row/v1";
  append_frame(b, "domain", dom, std::strlen(dom));
  append_frame(b, "field-name", F::kName, std::strlen(F::kName));
  u64("modulus", F::modulus_u64());
  u64("canonical-bytes", F::kBytes);
  u64("extension-degree", 1);
  const char* mode = "direct-interleaved-v1";
  append_frame(b, "decide-setup-mode", mode, std::strlen(mode));
  u64("level", s.level);
  u64("encoded-rows", s.encoded_rows);
  u64("message-rows", s.message_rows);
  u64("t-columns", s.t_cols);
  u64("t-elements", s.t_elements);
  u64("t-last-length", s.t_last_len);
  u64("h-columns", s.h_cols);
  return b;
}
template <class F>
Blake2s setup_row_hasher(const SetupShape& s, size_t row) {
  Blake2s h;
  h.update(setup_row_prefix<F>(s));
  absorb_framed_u64(h, "row", row);
  return h;
}
template <class F>
Digest hash_setup_row(const F* row, const SetupShape& s, size_t row_index) {
  Blake2s h = setup_row_hasher<F>(s, row_index);
  uint8_t e[F::kBytes];
  for (size_t c = 0; c < s.total_cols(); ++c) { row[c].to_bytes(e); h.update(e, F::kBytes); }
  return h.finalize();
}
template <class F>
MerkleTree build_setup_tree(const std::vector<F>& enc, const SetupShape& s) {
  s.validate();
  size_t cols = s.total_cols();
  if (enc.size() != s.encoded_rows * cols) fail(QF_E_ENCODING, "setup tree length");
  std::vector<Digest> leaves(s.encoded_rows);
#pragma omp parallel for if (s.encoded_rows >= 1024)
  for (long r = 0; r < long(s.encoded_rows); ++r) {
    std::vector<F> row(cols);
    for (size_t c = 0; c < cols; ++c) row[c] = enc[c * s.encoded_rows + r];
    leaves[r] = hash_setup_row<F>(row.data(), s, r);
  }
  return tree_from_leaves(std::move(leaves));
}

// Device acceleration of the setup commitments: encode_level fills a
// level's encoded matrix (column-major, encoded_rows x h_cols) and its row
// leaves (hash_setup_row), or returns false to leave the level to the host.
template <class F>
struct SetupAccel {
  virtual ~SetupAccel() {}
  virtual bool encode_level(const QaCode<F>& target, const QaCode<F>& current, size_t row_factor, const SetupShape& shape,
                            std::vector<F>& encoded, std::vector<Digest>& leaves) = 0;
};

template <class F>
struct PcsParams {
  size_t n_witness = 0, extension_columns = 0, index = 2, recursive_index = 2, security_bits = 0;
  double card_log2 = 0;
  QaSequence<F> seq;
  std::vector<std::unique_ptr<SetupLevel<F>>> setup;  // by level; [0] empty
  Digest derived_digest{}, setup_digest{}, parameter_digest{};

  size_t levels() const { return seq.codes.size(); }
  size_t top_rows() const { return seq.top().message_len; }
  size_t top_ext_rows() const { return seq.top().codeword_len(); }
  size_t base_columns() const { return extension_columns; }
  size_t num_queries(size_t level, size_t available) const {
    return seq.codes[level].num_queries(security_bits, available, card_log2);
  }
  const SetupLevel<F>& setup_level(size_t level) const {
    if (level >= setup.size() || !setup[level]) fail(QF_E_INVALID_COMMITMENT, "setup level");
    return *setup[level];
  }
};

template <class F>
double cardinality_log2() {
  return std::log2(double(F::cardinality()));
}

// ShortQaFoldPC::new_with_recursive_index + setup (qafold_short_pc.rs:358-444).
template <class F>
std::unique_ptr<PcsParams<F>> pcs_setup(size_t n_witness, size_t extension_columns, size_t security_bits, StdRng& rng,
                                        SetupAccel<F>* accel = nullptr) {
  auto pp = std::make_unique<PcsParams<F>>();
  pp->card_log2 = cardinality_log2<F>();
  size_t capacity_bits = size_t(std::floor(pp->card_log2 * 1.0));
  size_t max_bits = capacity_bits > 16 ? capacity_bits - 16 : 0;
  if (n_witness == 0 || !is_pow2(n_witness) || extension_columns <= 1 || !is_pow2(extension_columns) || security_bits == 0)
    fail(QF_E_ENCODING, "pcs parameters");
  if (security_bits > max_bits) fail(QF_E_INVALID_PARAMETERS, "requested soundness exceeds the short-field transcript limit");
  if (n_witness % extension_columns) fail(QF_E_ENCODING, "witness divisibility");
  pp->n_witness = n_witness;
  pp->extension_columns = extension_columns;
  pp->security_bits = security_bits;
  Digest seed;
  rng.fill_bytes(seed.data(), 32);
  pp->seq = build_sequence<F>(n_witness, extension_columns, seed);
  const size_t L = pp->seq.codes.size();
  // Derived parameters: DirectInterleavedV1 has no RFC sources.
  {
    Blake2s h;
    const char* dom = "qafold-short/derived-rfc-parameters/v1";
    absorb_framed(h, "domain", dom, std::strlen(dom));
    absorb_field_metadata<F>(h);
    const char* mode = "direct-interleaved-v1";
    absorb_framed(h, "decide-setup-mode", mode, std::strlen(mode));
    absorb_framed_u64(h, "levels", L);
    absorb_framed_u64(h, "switch-ratio", pp->seq.switch_ratio);
    uint8_t zero = 0;
    for (size_t level = 1; level < L; ++level) {
      absorb_framed_u64(h, "level", level);
      absorb_framed(h, "rfc-source-present", &zero, 1);
    }
    pp->derived_digest = h.finalize();
  }
  // Direct-interleaved setup commitments (qafold_short_setup.rs:427-536).
  pp->setup.resize(L);
  const size_t row_factor = pp->seq.switch_ratio;
  for (size_t level = 1; level < L; ++level) {
    const QaCode<F>& target = pp->seq.codes[level - 1];
    const QaCode<F>& current = pp->seq.codes[level];
    auto sl = std::make_unique<SetupLevel<F>>();
    sl->shape.level = level;
    sl->shape.encoded_rows = target.codeword_len();
    sl->shape.message_rows = target.message_len;
    sl->shape.h_cols = current.alphas.size() * row_factor;
    sl->shape.validate();
    std::vector<Digest> leaves;
    if (accel && accel->encode_level(target, current, row_factor, sl->shape, sl->encoded, leaves)) {
      if (sl->encoded.size() != sl->shape.encoded_rows * sl->shape.h_cols || leaves.size() != sl->shape.encoded_rows)
        fail(QF_E_ENCODING, "device setup level");
      sl->tree = tree_from_leaves(std::move(leaves));
    } else {
      const size_t er = sl->shape.encoded_rows, mr = sl->shape.message_rows;
      sl->encoded.assign(er * sl->shape.h_cols, F::zero());
#pragma omp parallel for schedule(dynamic)
      for (long col = 0; col < long(sl->shape.h_cols); ++col) {
        const auto& alpha = current.alphas[col / row_factor];
        size_t block = col % row_factor;
        target.encode_into(alpha.data() + block * mr, sl->encoded.data() + col * er);
      }
      sl->tree = build_setup_tree<F>(sl->encoded, sl->shape);
    }
    sl->root = sl->tree.root();
    pp->setup[level] = std::move(sl);
  }
  {
    Blake2s h;
    const char* dom = "qafold-short/setup-aggregate/v1";
    absorb_framed(h, "domain", dom, std::strlen(dom));
    absorb_field_metadata<F>(h);
    absorb_framed_u64(h, "levels", L);
    for (size_t level = 0; level < L; ++level) {
      absorb_framed_u64(h, "slot", level);
      uint8_t flag = level == 0 ? 0 : 1;
      absorb_framed(h, "present", &flag, 1);
      if (level > 0) {
        absorb_setup_shape(h, pp->setup[level]->shape);
        absorb_framed(h, "root", pp->setup[level]->root.data(), 32);
      }
    }
    pp->setup_digest = h.finalize();
  }
  {
    Blake2s h;
    const char* dom = "qafold-short-parameters/v4";
    absorb_framed(h, "domain", dom, std::strlen(dom));
    absorb_framed(h, "field-name", F::kName, std::strlen(F::kName));
    absorb_framed_u64(h, "modulus", F::modulus_u64());
    absorb_framed_u64(h, "extension-degree", 1);
    absorb_framed_u64(h, "witness", n_witness);
    absorb_framed_u64(h, "extension-columns", extension_columns);
    absorb_framed_u64(h, "index", 2);
    absorb_framed_u64(h, "security", security_bits);
    absorb_framed_u64(h, "rf-layers", pp->seq.rf_layers);
    absorb_framed(h, "generator-sequence", pp->seq.generator_digest.data(), 32);
    absorb_framed_u64(h, "recursive-index-override", 2);
    absorb_framed(h, "derived-rfc-sequence", pp->derived_digest.data(), 32);
    absorb_framed(h, "setup-roots-and-shapes", pp->setup_digest.data(), 32);
    pp->parameter_digest = h.finalize();
  }
  return pp;
}

// ------------------------------------------------------------ encoded matrices
// Read access to a committed column-major codeword (host- or device-resident).
template <class F>
struct CodewordView {
  virtual ~CodewordView() {}
  virtual Digest root() const = 0;
  virtual size_t ext_rows() const = 0;
  virtual size_t cols() const = 0;
  // Freivalds fold of the systematic half: out[r] = sum_c w[c] * entry(c, r), r < n_rows.
  virtual std::vector<F> fold_rows(size_t n_rows, const std::vector<F>& w) const = 0;
  // Row projection of the systematic half: out[c] = sum_r w[r] * entry(c, r), r < n_rows.
  virtual std::vector<F> project_rows(size_t n_rows, const std::vector<F>& w) const = 0;
  // Sampled rows and their authentication paths.
  virtual std::vector<std::vector<F>> rows(const std::vector<size_t>& idx) const = 0;
  virtual std::vector<std::vector<Digest>> paths(const std::vector<size_t>& idx) const = 0;
  // Every entry, column-major (all-row payloads of small codewords).
  virtual std::vector<F> entries() const = 0;
};

// A committed column-major codeword with its row tree, held on the host.
template <class F>
struct Codeword : CodewordView<F> {
  std::vector<F> encoded;  // encoded[col * n_ext_rows + row]
  size_t n_ext_rows = 0, n_cols = 0;
  MerkleTree tree;
  Digest root() const override { return tree.root(); }
  size_t ext_rows() const override { return n_ext_rows; }
  size_t cols() const override { return n_cols; }
  std::vector<F> row(size_t r) const {
    std::vector<F> v(n_cols);
    for (size_t c = 0; c < n_cols; ++c) v[c] = encoded[c * n_ext_rows + r];
    return v;
  }
  std::vector<F> fold_rows(size_t n_rows, const std::vector<F>& w) const override;
  std::vector<F> project_rows(size_t n_rows, const std::vector<F>& w) const override;
  std::vector<std::vector<F>> rows(const std::vector<size_t>& idx) const override {
    std::vector<std::vector<F>> out;
    for (size_t r : idx) out.push_back(row(r));
    return out;
  }
  std::vector<std::vector<Digest>> paths(const std::vector<size_t>& idx) const override {
    std::vector<std::vector<Digest>> out;
    for (size_t r : idx) out.push_back(tree.path(r));
    return out;
  }
  std::vector<F> entries() const override { return encoded; }
};

// Encode each message column and hash rows (commit_owned_inner and
// commit_extension_matrix differ only in the leaf domain).
template <class F>
Codeword<F> encode_and_commit(const QaCode<F>& code, const std::vector<F>& message, size_t n_cols, const char* domain) {
  const size_t R = code.message_len, R2 = code.codeword_len();
  if (message.size() != R * n_cols) fail(QF_E_ENCODING, "commit message length");
  Codeword<F> cw;
  cw.n_ext_rows = R2;
  cw.n_cols = n_cols;
  cw.encoded.assign(R2 * n_cols, F::zero());
#pragma omp parallel for schedule(dynamic)
  for (long c = 0; c < long(n_cols); ++c) code.encode_into(message.data() + c * R, cw.encoded.data() + c * R2);
  cw.tree = build_row_tree<F>(domain, cw.encoded, R2, n_cols);
  return cw;
}

// ------------------------------------------------------------ LiteBullet
template <class F>
struct LiteBullet {
  F a_value, b_value;
  std::vector<F> a_point, b_point;
};

template <class F>
LiteBullet<F> prove_litebullet(F claimed, std::vector<F> left, std::vector<F> right, PcsTranscript<F>& t, const char* label) {
  if (left.empty() || !is_pow2(left.size()) || left.size() != right.size() || inner_product(left, right) != claimed)
    fail(QF_E_INVALID_COMMITMENT, "litebullet claim");
  t.absorb_str("litebullet-domain", label);
  F rhs = claimed;
  LiteBullet<F> out;
  while (left.size() > 1) {
    size_t half = left.size() / 2;
    F lc = F::zero(), rc = F::zero();
    for (size_t i = 0; i < half; ++i) { lc += left[i] * right[half + i]; rc += left[half + i] * right[i]; }
    t.push_response(lc);
    t.push_response(rc);
    F ch = t.challenge_nonzero("litebullet-fold");
    F inv = ch.inverse();
    rhs += lc * ch + rc * inv;
    for (size_t i = 0; i < half; ++i) { left[i] += left[half + i] * inv; right[i] += right[half + i] * ch; }
    left.resize(half);
    right.resize(half);
    out.a_point.push_back(inv);
    out.b_point.push_back(ch);
  }
  out.a_value = left[0];
  out.b_value = right[0];
  t.push_response(out.a_value);
  t.push_response(out.b_value);
  if (out.a_value * out.b_value != rhs) fail(QF_E_INVALID_COMMITMENT, "litebullet terminal");
  return out;
}
template <class F>
std::optional<LiteBullet<F>> verify_litebullet(F claimed, size_t length, PcsTranscript<F>& t, const char* label) {
  if (length == 0 || !is_pow2(length)) return std::nullopt;
  t.absorb_str("litebullet-domain", label);
  F rhs = claimed;
  LiteBullet<F> out;
  size_t cur = length;
  while (cur > 1) {
    F lc = t.read_response();
    F rc = t.read_response();
    F ch = t.challenge_nonzero("litebullet-fold");
    F inv = ch.inverse();
    rhs += lc * ch + rc * inv;
    out.a_point.push_back(inv);
    out.b_point.push_back(ch);
    cur /= 2;
  }
  out.a_value = t.read_response();
  out.b_value = t.read_response();
  if (out.a_value * out.b_value != rhs) return std::nullopt;
  return out;
}

// ------------------------------------------------------------ rounds
template <class F>
struct VerifiedRound {
  F next_value;
  std::vector<F> next_point;
  F generator_value;
  std::vector<F> generator_left_point, generator_right_point;
  PendingH<F> pending(size_t level) const { return {level, generator_value, generator_left_point, generator_right_point}; }
};

template <class F>
void absorb_next_layer(PcsTranscript<F>& t, bool is_root, const Digest& d) {
  if (is_root) t.absorb_str("next-layer-kind", "extension-root");
  else t.absorb_str("next-layer-kind", "terminal-vector");
  t.absorb_digest("next-layer-binding", d);
}

template <class F>
VerifiedRound<F> prove_round_reductions(const QaCode<F>& code, const std::vector<F>& point, const std::vector<F>& freivalds,
                                        F freivalds_value, const std::vector<F>& folded, const std::vector<F>& row_weights,
                                        const RowSelection& sel, const std::vector<F>& sampled, PcsTranscript<F>& t) {
  const size_t n_rows = code.message_len, n_ext = code.codeword_len();
  const size_t col_log = ilog2(freivalds.size());
  if (point.size() != col_log + size_t(ilog2(n_rows)) || folded.size() != n_rows || row_weights.size() != n_rows ||
      sel.size() != sampled.size())
    fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "round reduction dims");
  size_t sel_log = ilog2(next_pow2(sel.size()));
  std::vector<F> sel_point;
  for (size_t i = 0; i < sel_log; ++i) sel_point.push_back(t.challenge_ext("selection-left"));
  std::vector<F> sw = tensor_weights_prefix(sel_point, sel.size());
  F selected_value = inner_product(sw, sampled);
  std::vector<F> pi_left(n_ext, F::zero());
  for (size_t i = 0; i < sel.size(); ++i) pi_left[sel.at(i)] += sw[i];
  std::vector<F> combined_left = code.generator_left_projection(pi_left);
  F rho = t.challenge_ext("opening-batch");
  F combined_value = selected_value + rho * freivalds_value;
  for (size_t i = 0; i < n_rows; ++i) combined_left[i] += rho * row_weights[i];
  LiteBullet<F> msg = prove_litebullet<F>(combined_value, std::move(combined_left), folded, t, "message-litebullet");
  std::vector<F> pt_rows(point.begin() + col_log, point.end());
  F opening_left_eval = tensor_inner_product(pt_rows, msg.a_point);
  F selection_left_eval = msg.a_value - rho * opening_left_eval;
  std::vector<F> gen_right = code.generator_right_projection(tensor_weights(msg.a_point));
  LiteBullet<F> gen = prove_litebullet<F>(selection_left_eval, std::move(pi_left), std::move(gen_right), t, "generator-litebullet");
  return {msg.b_value, msg.b_point, gen.b_value, gen.b_point, msg.a_point};
}

template <class F>
std::optional<VerifiedRound<F>> verify_round_reductions(const QaCode<F>& code, const std::vector<F>& point, size_t n_cols,
                                                        F freivalds_value, const RowSelection& sel,
                                                        const std::vector<F>& sampled, PcsTranscript<F>& t) {
  const size_t n_rows = code.message_len, n_ext = code.codeword_len();
  const size_t col_log = ilog2(n_cols);
  if (n_cols == 0 || !is_pow2(n_cols) || point.size() != col_log + size_t(ilog2(n_rows)) || sel.size() != sampled.size())
    return std::nullopt;
  size_t sel_log = ilog2(next_pow2(sel.size()));
  std::vector<F> sel_point;
  for (size_t i = 0; i < sel_log; ++i) sel_point.push_back(t.challenge_ext("selection-left"));
  std::vector<F> sw = tensor_weights_prefix(sel_point, sel.size());
  F selected_value = inner_product(sw, sampled);
  F rho = t.challenge_ext("opening-batch");
  F combined_value = selected_value + rho * freivalds_value;
  auto msg = verify_litebullet<F>(combined_value, n_rows, t, "message-litebullet");
  if (!msg) return std::nullopt;
  std::vector<F> pt_rows(point.begin() + col_log, point.end());
  F opening_left_eval = tensor_inner_product(pt_rows, msg->a_point);
  F selection_left_eval = msg->a_value - rho * opening_left_eval;
  auto gen = verify_litebullet<F>(selection_left_eval, n_ext, t, "generator-litebullet");
  if (!gen) return std::nullopt;
  F expected = F::zero();
  for (size_t i = 0; i < sel.size(); ++i) expected += sw[i] * tensor_weight_at(gen->a_point, sel.at(i));
  if (gen->a_value != expected) return std::nullopt;
  return VerifiedRound<F>{msg->b_value, msg->b_point, gen->b_value, gen->b_point, msg->a_point};
}

template <class F>
std::vector<F> Codeword<F>::project_rows(size_t n_rows, const std::vector<F>& w) const {
  std::vector<F> out(n_cols, F::zero());
#pragma omp parallel for if (n_rows >= 4096)
  for (long c = 0; c < long(n_cols); ++c) {
    F s = F::zero();
    const F* col = encoded.data() + c * n_ext_rows;
    for (size_t r = 0; r < n_rows; ++r) s += w[r] * col[r];
    out[c] = s;
  }
  return out;
}
template <class F>
std::vector<F> Codeword<F>::fold_rows(size_t n_rows, const std::vector<F>& weights) const {
  std::vector<F> out(n_rows);
#pragma omp parallel for if (n_rows >= 4096)
  for (long r = 0; r < long(n_rows); ++r) {
    F s = F::zero();
    for (size_t c = 0; c < n_cols; ++c) s += weights[c] * encoded[c * n_ext_rows + r];
    out[r] = s;
  }
  return out;
}
template <class F>
std::vector<F> systematic_row_projection(const CodewordView<F>& cw, size_t n_rows, const std::vector<F>& w) {
  return cw.project_rows(n_rows, w);
}

// One opening round (top or extension).  `next` is the next code, or null at
// the last level.  The caller has checked/absorbed the opening vector input.
template <class F>
struct RoundOutput {
  Rows<F> rows;
  std::optional<std::vector<F>> terminal;
  VerifiedRound<F> reduction;
  std::unique_ptr<CodewordView<F>> next_cw;
};

// Runs the top opening round with its message-length vectors (the Freivalds
// fold, the next-level commitment, the generator projections and both
// LiteBullets) resident on a device.  Same transcript and outputs as
// prove_round; `opening` is the top row projection.
template <class F>
struct TopRoundAccel {
  virtual ~TopRoundAccel() {}
  virtual RoundOutput<F> prove_top_round(const PcsParams<F>& pp, size_t level, const std::vector<F>& point,
                                         const std::vector<F>& opening, PcsTranscript<F>& t) = 0;
  // For a codeword produced by this accelerator: computes the extension
  // round's opening vector on the device and returns true, after which
  // prove_top_round runs the round; false keeps the round on the host.
  virtual bool open_round(const CodewordView<F>& cw, size_t n_rows, const std::vector<F>& point, size_t col_log,
                          std::vector<F>& opening) {
    return false;
  }
};

template <class F>
RoundOutput<F> prove_round(const PcsParams<F>& pp, size_t level, const CodewordView<F>& cw, const std::vector<F>& point,
                           const std::vector<F>& opening, const std::vector<F>& row_weights, PcsTranscript<F>& t) {
  const QaCode<F>& code = pp.seq.codes[level];
  const QaCode<F>* next = level > 0 ? &pp.seq.codes[level - 1] : nullptr;
  const size_t n_rows = code.message_len, n_cols = cw.cols(), n_ext = cw.ext_rows();
  t.absorb_digest("round-root", cw.root());
  for (const F& o : opening) t.push_response(o);
  std::vector<F> freivalds;
  for (size_t i = 0; i < n_cols; ++i) freivalds.push_back(t.challenge_ext("freivalds"));
  F freivalds_value = inner_product(opening, freivalds);
  std::vector<F> folded = cw.fold_rows(n_rows, freivalds);
  RoundOutput<F> out;
  if (next) {
    // Folded vector is the next level's column-major message (32 columns).
    out.next_cw = std::make_unique<Codeword<F>>(encode_and_commit(*next, folded, pp.extension_columns, kLeafExtDomain));
    absorb_next_layer(t, true, out.next_cw->root());
  } else {
    absorb_next_layer(t, false, hash_terminal_vector(folded));
  }
  size_t qc = pp.num_queries(level, n_ext);
  Digest seed = t.challenge_digest("row-selection");
  RowSelection sel = make_selection(qc, n_ext, seed);
  std::vector<F> sampled(sel.size());
  if (sel.all) {
    std::vector<F> all = cw.entries();
    for (size_t r = 0; r < n_ext; ++r) {
      F s = F::zero();
      for (size_t c = 0; c < n_cols; ++c) s += freivalds[c] * all[c * n_ext + r];
      sampled[r] = s;
    }
    out.rows.all = true;
    out.rows.n_rows = n_ext;
    out.rows.n_cols = n_cols;
    out.rows.encoded = std::move(all);
  } else {
    std::vector<std::vector<F>> rws = cw.rows(sel.rows);
    std::vector<std::vector<Digest>> pths = cw.paths(sel.rows);
    for (size_t i = 0; i < sel.size(); ++i) {
      RowQuery<F> q;
      q.row = std::move(rws[i]);
      q.path.siblings = std::move(pths[i]);
      F s = F::zero();
      for (size_t c = 0; c < n_cols; ++c) s += freivalds[c] * q.row[c];
      sampled[i] = s;
      out.rows.partial.push_back(std::move(q));
    }
  }
  t.absorb_exts("sampled-values", sampled);
  out.reduction = prove_round_reductions(code, point, freivalds, freivalds_value, folded, row_weights, sel, sampled, t);
  if (!next) out.terminal = std::move(folded);
  return out;
}

template <class F>
struct OpenResult {
  F claimed;
  OpeningProof<F> proof;
  Reduction<F> reduction;
};

// open_with_reduction (qafold_short_pc.rs:578-730).  `opening` is the top row
// projection (computed by the caller's backend) and `claimed` its value.
template <class F>
OpenResult<F> open_with_reduction(const PcsParams<F>& pp, const CodewordView<F>& top, const std::vector<F>& point,
                                  const std::vector<F>& opening, F claimed, const std::vector<F>& row_weights,
                                  TopRoundAccel<F>* accel = nullptr) {
  if (point.size() != size_t(ilog2(pp.n_witness))) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "opening point length");
  PcsTranscript<F> t;
  t.absorb_digest("parameters", pp.parameter_digest);
  t.absorb_digest("commitment", top.root());
  t.absorb_exts("point", point);
  t.absorb_ext("claimed-value", claimed);
  const size_t L = pp.levels(), top_level = L - 1;
  OpenResult<F> res;
  res.claimed = claimed;
  RoundOutput<F> r0 = accel ? accel->prove_top_round(pp, top_level, point, opening, t)
                            : prove_round(pp, top_level, top, point, opening, row_weights, t);
  res.proof.top = std::move(r0.rows);
  if (top_level == 0) {
    if (evaluate_generator_mle(pp.seq.codes[0], r0.reduction.generator_left_point, r0.reduction.generator_right_point) !=
        r0.reduction.generator_value)
      fail(QF_E_INVALID_COMMITMENT, "top generator claim");
  } else {
    res.reduction.pending.push_back(r0.reduction.pending(top_level));
  }
  F next_value = r0.reduction.next_value;
  std::vector<F> next_point = r0.reduction.next_point;
  std::optional<std::vector<F>> terminal = std::move(r0.terminal);
  std::unique_ptr<CodewordView<F>> prepared = std::move(r0.next_cw);
  const size_t col_log = ilog2(pp.extension_columns);
  for (size_t level = top_level; level-- > 0;) {
    if (terminal || !prepared) fail(QF_E_ENCODING, "round sequencing");
    const QaCode<F>& code = pp.seq.codes[level];
    std::vector<F> rw, opening_vec;
    const bool on_device = accel && accel->open_round(*prepared, code.message_len, next_point, col_log, opening_vec);
    if (!on_device) {
      rw = tensor_weights(std::vector<F>(next_point.begin() + col_log, next_point.end()));
      opening_vec = systematic_row_projection(*prepared, code.message_len, rw);
    }
    std::vector<F> cw_pt(next_point.begin(), next_point.begin() + col_log);
    if (inner_product(opening_vec, tensor_weights(cw_pt)) != next_value) fail(QF_E_INVALID_COMMITMENT, "extension opening");
    RoundOutput<F> r;
    if (on_device) {
      r = accel->prove_top_round(pp, level, next_point, opening_vec, t);
    } else {
      Section sec("opening_round_host");
      r = prove_round(pp, level, *prepared, next_point, opening_vec, rw, t);
    }
    res.proof.ext_rounds.push_back(ExtRound<F>{prepared->root(), std::move(r.rows)});
    if (level == 0) {
      if (evaluate_generator_mle(code, r.reduction.generator_left_point, r.reduction.generator_right_point) !=
          r.reduction.generator_value)
        fail(QF_E_INVALID_COMMITMENT, "base generator claim");
    } else {
      res.reduction.pending.push_back(r.reduction.pending(level));
    }
    terminal = std::move(r.terminal);
    next_value = r.reduction.next_value;
    next_point = r.reduction.next_point;
    prepared = std::move(r.next_cw);
  }
  F ev;
  if (!terminal || prepared || terminal->empty() || !is_pow2(terminal->size()) ||
      next_point.size() != size_t(ilog2(terminal->size())) || !mle_eval(*terminal, next_point, ev) || ev != next_value)
    fail(QF_E_INVALID_COMMITMENT, "terminal vector");
  res.proof.responses = std::move(t.responses);
  res.proof.base_vector = std::move(*terminal);
  res.reduction.ok = true;
  return res;
}

// Authenticates rows and returns the Freivalds-combined sampled values.
template <class F>
std::optional<std::vector<F>> authenticate_rows(const Rows<F>& rows, const RowSelection& sel, size_t n_ext_rows, size_t n_cols,
                                                const Digest& root, const std::vector<F>& freivalds, const char* domain) {
  std::vector<F> sampled;
  if (!rows.all) {
    if (sel.all || rows.partial.size() != sel.size()) return std::nullopt;
    for (size_t i = 0; i < rows.partial.size(); ++i) {
      const auto& q = rows.partial[i];
      if (q.row.size() != n_cols) return std::nullopt;
      Digest leaf = hash_row<F>(domain, q.row.data(), n_cols);
      if (!verify_merkle_siblings(leaf, sel.at(i), n_ext_rows, q.path.siblings, root)) return std::nullopt;
      F s = F::zero();
      for (size_t c = 0; c < n_cols; ++c) s += freivalds[c] * q.row[c];
      sampled.push_back(s);
    }
    return sampled;
  }
  if (!sel.all || sel.size() != n_ext_rows || rows.n_rows != n_ext_rows || rows.n_cols != n_cols ||
      rows.encoded.size() != n_ext_rows * n_cols)
    return std::nullopt;
  if (build_row_tree<F>(domain, rows.encoded, n_ext_rows, n_cols).root() != root) return std::nullopt;
  for (size_t r = 0; r < n_ext_rows; ++r) {
    F s = F::zero();
    for (size_t c = 0; c < n_cols; ++c) s += freivalds[c] * rows.encoded[c * n_ext_rows + r];
    sampled.push_back(s);
  }
  return sampled;
}

template <class F>
std::optional<VerifiedRound<F>> verify_round(const PcsParams<F>& pp, size_t level, const Digest& root, size_t n_cols,
                                             const std::vector<F>& point, F value, bool next_is_root,
                                             const Digest& next_binding, const Rows<F>& rows, const char* domain,
                                             PcsTranscript<F>& t) {
  const QaCode<F>& code = pp.seq.codes[level];
  const size_t n_rows = code.message_len, n_ext = code.codeword_len();
  const size_t col_log = ilog2(n_cols);
  if (point.size() != col_log + size_t(ilog2(n_rows))) return std::nullopt;
  t.absorb_digest("round-root", root);
  std::vector<F> opening;
  for (size_t i = 0; i < n_cols; ++i) opening.push_back(t.read_response());
  std::vector<F> cw_pt(point.begin(), point.begin() + col_log);
  if (inner_product(opening, tensor_weights(cw_pt)) != value) return std::nullopt;
  std::vector<F> freivalds;
  for (size_t i = 0; i < n_cols; ++i) freivalds.push_back(t.challenge_ext("freivalds"));
  F fv = inner_product(opening, freivalds);
  absorb_next_layer(t, next_is_root, next_binding);
  size_t qc = pp.num_queries(level, n_ext);
  Digest seed = t.challenge_digest("row-selection");
  RowSelection sel = make_selection(qc, n_ext, seed);
  auto sampled = authenticate_rows(rows, sel, n_ext, n_cols, root, freivalds, domain);
  if (!sampled) return std::nullopt;
  t.absorb_exts("sampled-values", *sampled);
  return verify_round_reductions(code, point, n_cols, fv, sel, *sampled, t);
}

// verify_opening_reduction (qafold_short_pc.rs:736-864).
template <class F>
Reduction<F> verify_opening_reduction(const PcsParams<F>& pp, const Digest& root, const std::vector<F>& point, F claimed,
                                      const OpeningProof<F>& proof) {
  Reduction<F> rejected;
  const size_t L = pp.levels();
  if (point.size() != size_t(ilog2(pp.n_witness)) || proof.ext_rounds.size() != L - 1) return rejected;
  PcsTranscript<F> t(&proof.responses);
  t.absorb_digest("parameters", pp.parameter_digest);
  t.absorb_digest("commitment", root);
  t.absorb_exts("point", point);
  t.absorb_ext("claimed-value", claimed);
  const size_t top_level = L - 1;
  Reduction<F> out;
  bool next_root = top_level != 0;
  Digest nb = next_root ? proof.ext_rounds[0].root : hash_terminal_vector(proof.base_vector);
  auto top = verify_round(pp, top_level, root, pp.extension_columns, point, claimed, next_root, nb, proof.top, kLeafBaseDomain, t);
  if (!top) return rejected;
  if (top_level == 0) {
    if (evaluate_generator_mle(pp.seq.codes[0], top->generator_left_point, top->generator_right_point) != top->generator_value)
      return rejected;
  } else {
    out.pending.push_back(top->pending(top_level));
  }
  F expected = top->next_value;
  std::vector<F> cur = top->next_point;
  size_t ri = 0;
  for (size_t level = top_level; level-- > 0; ++ri) {
    const auto& pr = proof.ext_rounds[ri];
    bool nr = ri + 1 < proof.ext_rounds.size();
    Digest b = nr ? proof.ext_rounds[ri + 1].root : hash_terminal_vector(proof.base_vector);
    auto red = verify_round(pp, level, pr.root, pp.extension_columns, cur, expected, nr, b, pr.rows, kLeafExtDomain, t);
    if (!red) return rejected;
    if (level == 0) {
      if (evaluate_generator_mle(pp.seq.codes[0], red->generator_left_point, red->generator_right_point) != red->generator_value)
        return rejected;
    } else {
      out.pending.push_back(red->pending(level));
    }
    expected = red->next_value;
    cur = red->next_point;
  }
  F ev;
  if (proof.base_vector.empty() || !is_pow2(proof.base_vector.size()) || cur.size() != size_t(ilog2(proof.base_vector.size())) ||
      !mle_eval(proof.base_vector, cur, ev) || ev != expected)
    return rejected;
  out.ok = t.exhausted();
  return out;
}

}  // namespace qf
