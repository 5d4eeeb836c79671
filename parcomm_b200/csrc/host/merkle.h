// BLAKE2s Merkle trees over encoded rows, and the PCS framed transcript.
//
// Reference: leaf/inner domains and framing (qafold_short_pc.rs:24-33,
// 2372-2517), Blake2sMerkleTree and paths (978-1021), verify_merkle_siblings
// (1859-1893), ShortTranscriptWriter/Reader with derive_digest and
// derive_extension_challenge (2012-2230), sample_without_replacement /
// sample_below (3000-3047).
#pragma once
#include <map>
#include <vector>

#include "blake2s.h"
#include "qacode.h"

namespace qf {

static const char* kLeafBaseDomain = "qafold-short/base-row/v1";
static const char* kLeafExtDomain = "qafold-short/extension-row/v1";
static const char* kInnerDomain = "qafold-short/merkle-inner/v1";
static const char* kTerminalVectorDomain = "qafold-short/terminal-vector/v1";
static const char* kTranscriptDomain = "brakefold/qafold-short-pcs/v2";

inline Digest hash_inner(const Digest& l, const Digest& r) {
  Blake2s h;
  absorb_framed(h, "domain", kInnerDomain, std::strlen(kInnerDomain));
  h.update(l);
  h.update(r);
  return h.finalize();
}

// Hash of one encoded row: frame(domain) || frame(width) || canonical values.
template <class F>
Digest hash_row(const char* domain, const F* row, size_t n_cols) {
  Blake2s h;
  absorb_framed(h, "domain", domain, std::strlen(domain));
  absorb_framed_u64(h, "width", n_cols);
  uint8_t enc[F::kBytes];
  for (size_t c = 0; c < n_cols; ++c) { row[c].to_bytes(enc); h.update(enc, F::kBytes); }
  return h.finalize();
}

struct MerkleTree {
  std::vector<std::vector<Digest>> levels;  // levels[0] = leaves
  Digest root() const { return levels.empty() ? Digest{} : levels.back()[0]; }
  size_t leaves() const { return levels.empty() ? 0 : levels[0].size(); }
  std::vector<Digest> path(size_t index) const {
    if (index >= leaves()) fail(QF_E_INVALID_COMMITMENT, "merkle path index");
    std::vector<Digest> sib;
    for (size_t l = 0; l + 1 < levels.size(); ++l) { sib.push_back(levels[l][index ^ 1]); index >>= 1; }
    return sib;
  }
};

inline MerkleTree tree_from_leaves(std::vector<Digest> leaves) {
  if (leaves.empty() || !is_pow2(leaves.size())) fail(QF_E_ENCODING, "merkle leaves");
  MerkleTree t;
  t.levels.push_back(std::move(leaves));
  while (t.levels.back().size() > 1) {
    const auto& c = t.levels.back();
    std::vector<Digest> p(c.size() / 2);
#pragma omp parallel for if (p.size() >= 4096)
    for (long i = 0; i < long(p.size()); ++i) p[i] = hash_inner(c[2 * i], c[2 * i + 1]);
    t.levels.push_back(std::move(p));
  }
  return t;
}

// Column-major encoded matrix entries[col * n_rows + row] -> row-leaf tree.
template <class F>
MerkleTree build_row_tree(const char* domain, const std::vector<F>& entries, size_t n_rows, size_t n_cols) {
  if (n_rows == 0 || !is_pow2(n_rows) || n_cols == 0 || entries.size() != n_rows * n_cols)
    fail(QF_E_ENCODING, "row tree shape");
  std::vector<Digest> leaves(n_rows);
#pragma omp parallel for if (n_rows >= 4096)
  for (long r = 0; r < long(n_rows); ++r) {
    std::vector<F> row(n_cols);
    for (size_t c = 0; c < n_cols; ++c) row[c] = entries[c * n_rows + r];
    leaves[r] = hash_row<F>(domain, row.data(), n_cols);
  }
  return tree_from_leaves(std::move(leaves));
}

inline bool verify_merkle_siblings(Digest digest, size_t index, size_t leaf_count, const std::vector<Digest>& sib,
                                   const Digest& root) {
  if (leaf_count == 0 || !is_pow2(leaf_count) || index >= leaf_count || sib.size() != size_t(ilog2(leaf_count)))
    return false;
  for (const Digest& s : sib) {
    digest = (index & 1) == 0 ? hash_inner(digest, s) : hash_inner(s, digest);
    index >>= 1;
  }
  return digest == root;
}

template <class F>
Digest hash_terminal_vector(const std::vector<F>& values) {
  Blake2s h;
  absorb_framed(h, "domain", kTerminalVectorDomain, std::strlen(kTerminalVectorDomain));
  absorb_framed_u64(h, "length", values.size());
  uint8_t enc[F::kBytes];
  for (const F& v : values) { v.to_bytes(enc); absorb_framed(h, "element", enc, F::kBytes); }
  return h.finalize();
}

// ---------------------------------------------------------------- transcript
inline Digest derive_digest(const Blake2s& state, const char* label, uint64_t counter, uint64_t coeff, uint64_t attempt) {
  Blake2s h = state;
  absorb_framed(h, "challenge-label", label, std::strlen(label));
  h.update_u64(counter);
  h.update_u64(coeff);
  h.update_u64(attempt);
  return h.finalize();
}

// Writer and reader share all absorption logic; the reader replays responses.
template <class F>
struct PcsTranscript {
  Blake2s hasher;
  uint64_t counter = 0;
  std::vector<F> responses;        // writer output
  const std::vector<F>* replay = nullptr;  // reader input
  size_t cursor = 0;

  PcsTranscript() { absorb_bytes("domain", kTranscriptDomain, std::strlen(kTranscriptDomain)); }
  explicit PcsTranscript(const std::vector<F>* r) : PcsTranscript() { replay = r; }
  bool reading() const { return replay != nullptr; }

  void absorb_bytes(const char* label, const void* b, size_t n) { absorb_framed(hasher, label, b, n); }
  void absorb_str(const char* label, const char* s) { absorb_bytes(label, s, std::strlen(s)); }
  void absorb_u64(const char* label, uint64_t v) { auto b = le64(v); absorb_bytes(label, b.data(), 8); }
  void absorb_u8(const char* label, uint8_t v) { absorb_bytes(label, &v, 1); }
  void absorb_digest(const char* label, const Digest& d) { absorb_bytes(label, d.data(), 32); }
  void absorb_ext(const char* label, const F& v) { uint8_t e[F::kBytes]; v.to_bytes(e); absorb_bytes(label, e, F::kBytes); }
  void absorb_exts(const char* label, const std::vector<F>& vs) {
    absorb_bytes("vector-label", label, std::strlen(label));
    absorb_u64("vector-length", vs.size());
    for (const F& v : vs) absorb_ext("vector-element", v);
  }
  // Writer: push a prover message.  Reader: the same call reads it back.
  F response(const F& v_if_writing = F::zero()) {
    F v = v_if_writing;
    if (reading()) {
      if (cursor >= replay->size()) fail(QF_E_TRANSCRIPT, "transcript responses exhausted");
      v = (*replay)[cursor++];
    } else {
      responses.push_back(v);
    }
    absorb_ext("response", v);
    return v;
  }
  void push_response(const F& v) { response(v); }
  F read_response() { return response(); }
  bool exhausted() const { return reading() && cursor == replay->size(); }

  Digest challenge_digest(const char* label) {
    Digest d = derive_digest(hasher, label, counter, 0, 0);
    ++counter;
    absorb_str("digest-challenge-label", label);
    absorb_digest("digest-challenge", d);
    return d;
  }
  F challenge_ext_impl(const char* label, bool nonzero) {
    uint64_t c = counter;
    for (uint64_t outer = 0;; ++outer) {
      // EXTENSION_DEGREE = 1: one coefficient, attempts continue from `outer`.
      F value;
      for (uint64_t attempt = outer;; ++attempt) {
        Digest d = derive_digest(hasher, label, c, 0, attempt);
        if (F::from_uniform_bytes(d.data(), value)) break;
      }
      if (!nonzero || !value.is_zero()) {
        ++counter;
        absorb_str("field-challenge-label", label);
        absorb_ext("field-challenge", value);
        return value;
      }
    }
  }
  F challenge_ext(const char* label) { return challenge_ext_impl(label, false); }
  F challenge_nonzero(const char* label) { return challenge_ext_impl(label, true); }
};

inline size_t sample_below(const Digest& seed, uint64_t& counter, size_t upper) {
  if (upper == 0) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "sample_below");
  unsigned __int128 range = (unsigned __int128)1 << 64;
  unsigned __int128 limit = range - range % upper;
  for (;;) {
    Blake2s h;
    h.update_str("qafold-short-index/v1");
    h.update(seed);
    h.update_u64(counter);
    ++counter;
    Digest d = h.finalize();
    uint64_t cand = 0;
    for (int i = 0; i < 8; ++i) cand |= uint64_t(d[i]) << (8 * i);
    if ((unsigned __int128)cand < limit) return size_t(cand % upper);
  }
}

inline std::vector<size_t> sample_without_replacement(size_t count, size_t population, const Digest& seed) {
  if (count == 0 || count > population) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "sample count");
  std::vector<size_t> out;
  if (count == population) { for (size_t i = 0; i < population; ++i) out.push_back(i); return out; }
  std::map<size_t, size_t> swaps;
  uint64_t counter = 0;
  for (size_t off = 0; off < count; ++off) {
    size_t remaining = population - off;
    size_t s = sample_below(seed, counter, remaining);
    size_t last = remaining - 1;
    auto it = swaps.find(s);
    size_t sv = it == swaps.end() ? s : it->second;
    auto jt = swaps.find(last);
    size_t lv = jt == swaps.end() ? last : jt->second;
    swaps[s] = lv;
    out.push_back(sv);
  }
  return out;
}

// Row selection: all rows, or a sampled partial list.
struct RowSelection {
  bool all = false;
  size_t count = 0;
  std::vector<size_t> rows;
  size_t size() const { return all ? count : rows.size(); }
  size_t at(size_t i) const { return all ? i : rows[i]; }
};
inline RowSelection make_selection(size_t query_count, size_t available, const Digest& seed) {
  if (query_count == 0 || query_count > available) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "selection");
  RowSelection s;
  if (query_count == available) { s.all = true; s.count = available; }
  else s.rows = sample_without_replacement(query_count, available, seed);
  return s;
}

}  // namespace qf
