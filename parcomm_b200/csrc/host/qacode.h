// Systematic index-two QA codes over a full extension field, the geometric
// code sequence, and the f64 distance / query-count policy.
//
// Reference: ShortQaCode (qafold_short.rs:664-1207), ShortQaFold
// (qafold_short.rs:1641-1895), unnormalised WHT (1911-2016),
// derive_level_seed / sample_generator_element / generator digests
// (2211-2325), QA distance bounds (qafold.rs:27-178) and query counts
// (brakefold.rs:4-17).  Both supported fields use EXTENSION_DEGREE = 1,
// DirectInterleavedV1 setup and finite-length proximity
// (full_extension.rs:120-130, koalabear.rs:195-202), so the RF-code and
// nonzero-frequency branches of the reference are not reachable and are not
// restated here.
#pragma once
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <stdexcept>
#include <tuple>
#include <string>
#include <vector>

#include "blake2s.h"

namespace qf {

struct QfError : std::runtime_error {
  int code;
  QfError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
// Error codes mirror mikros_qafold::Error (vendor lib.rs:20-35) plus the
// protocol's static `check` strings.
#ifndef QF_OK  // same values as include/parcomm_qafold.h
#define QF_OK 0
#define QF_E_ENCODING -1
#define QF_E_HASHING -2
#define QF_E_INVALID_COMMITMENT -3
#define QF_E_INVALID_NUMBER_OF_VARIABLES -4
#define QF_E_INVALID_PARAMETERS -5
#define QF_E_TRANSCRIPT -6
#define QF_E_PROTOCOL -7
#define QF_E_CUDA -8
#define QF_E_ARGUMENT -9
#define QF_E_NO_DEVICE -10
#endif
[[noreturn]] inline void fail(int code, const std::string& msg) { throw QfError(code, msg); }
inline void check(bool ok, const char* msg) { if (!ok) fail(QF_E_PROTOCOL, msg); }

inline bool is_pow2(uint64_t x) { return x && !(x & (x - 1)); }
inline int ilog2(uint64_t x) { return 63 - __builtin_clzll(x); }
inline uint64_t next_pow2(uint64_t x) { return x <= 1 ? 1 : (uint64_t(1) << (64 - __builtin_clzll(x - 1))); }

// ---------------------------------------------------------------- WHT
// Unnormalised Walsh-Hadamard transform, (a, b) -> (a + b, a - b), natural
// order.  Any stage order gives the same exact result.
template <class F>
void wht_in_place(F* v, size_t n) {
  // Butterfly k of a level pairs i = (k / half) * 2 half + k % half with
  // i + half; large transforms spread each level over the OpenMP threads.
  for (size_t half = 1, lh = 0; half < n; half <<= 1, ++lh) {
#pragma omp parallel for schedule(static) if (n >= (size_t(1) << 18))
    for (long k = 0; k < long(n / 2); ++k) {
      const size_t i = ((size_t(k) >> lh) << (lh + 1)) | (size_t(k) & (half - 1));
      F a = v[i], b = v[i + half];
      v[i] = a + b;
      v[i + half] = a - b;
    }
  }
}

// ---------------------------------------------------------------- distances
namespace dist {
inline double log_one_minus_exp(double x, bool& ok) {
  if (x >= 0.0) { ok = false; return 0; }
  ok = true;
  if (x < -M_LN2) return std::log1p(-std::exp(x));
  return std::log(-std::expm1(x));
}
inline double log_add_exp(double a, double b) {
  double m = a > b ? a : b;  // f64::max (neither is NaN here)
  return m + std::log(std::exp(a - m) + std::exp(b - m));
}
inline bool qa_epsilon_at(size_t message_len, size_t index, double distance, double ln_p, double& eps) {
  if (message_len == 0 || index <= 1 || !(distance > 0.0 && distance < 1.0) || !(ln_p > 0.0)) return false;
  double ln_p_minus_one = ln_p + std::log1p(-std::exp(-ln_p));
  double g = 1.0 - distance * ln_p_minus_one / ln_p + distance * std::log(distance) / ln_p +
             (1.0 - distance) * std::log(1.0 - distance) / ln_p;
  double epsilon = g - (1.0 + std::log(double(message_len)) / ln_p) / double(index);
  if (epsilon > 0.0) { eps = epsilon; return true; }
  return false;
}
inline bool qa_bound_at(size_t message_len, size_t index, double distance, double ln_p, double& eps_out, double& logf) {
  double epsilon;
  if (!qa_epsilon_at(message_len, index, distance, ln_p, epsilon)) return false;
  double ln_p_minus_one = ln_p + std::log1p(-std::exp(-ln_p));
  bool ok;
  double lome = log_one_minus_exp(-double(index) * epsilon * ln_p, ok);
  if (!ok) return false;
  double denominator_log = lome + ln_p_minus_one;
  double first_collision = double(index) * double(index - 1) * double(message_len) / 2.0;
  double first_collision_log = std::log(first_collision) - 2.0 * ln_p;
  double first_exponent = std::ceil(double(index - 1) / (double(index) * distance)) * double(index) * epsilon;
  double first_tail_log = -first_exponent * ln_p - denominator_log;
  double first_failure_log = log_add_exp(first_collision_log, first_tail_log);
  double second_collision_log = std::log(double(index) * double(message_len)) - ln_p;
  double second_exponent = std::ceil(1.0 / distance) * double(index) * epsilon;
  double second_tail_log = -second_exponent * ln_p - denominator_log;
  double second_failure_log = log_add_exp(second_collision_log, second_tail_log);
  eps_out = epsilon;
  logf = first_failure_log < second_failure_log ? first_failure_log : second_failure_log;
  return true;
}
// qafold.rs:75-131.  Returns false for "InvalidParameters" (no admissible distance).
inline bool qa_distance_bound_uncached(size_t message_len, size_t index, size_t security_bits, double modulus_log2, double& rel) {
  if (message_len == 0 || !is_pow2(message_len) || index <= 1 || !is_pow2(index) || security_bits == 0 ||
      !std::isfinite(modulus_log2) || modulus_log2 <= 0.0)
    fail(QF_E_ENCODING, "qa distance arguments");
  double ln_p = modulus_log2 * M_LN2;
  double upper = 1.0 - 1.0 / double(index);
  double target = -double(security_bits) * M_LN2;
  auto valid = [&](double d) {
    double e, lf;
    return qa_bound_at(message_len, index, d, ln_p, e, lf) && lf <= target;
  };
  const size_t scan_steps = 4096;
  double lower = 0.0, upper_bracket = upper;
  for (size_t step = 1; step <= scan_steps; ++step) {
    double candidate = upper * double(step) / double(scan_steps);
    if (valid(candidate)) lower = candidate;
    else if (candidate > lower) { upper_bracket = candidate; break; }
  }
  if (lower == 0.0) return false;
  for (int i = 0; i < 96; ++i) {
    double middle = (lower + upper_bracket) * 0.5;
    if (valid(middle)) lower = middle; else upper_bracket = middle;
  }
  double relative = lower * (1.0 - 1e-12);
  double e, lf;
  if (!qa_bound_at(message_len, index, relative, ln_p, e, lf)) fail(QF_E_ENCODING, "qa bound");
  rel = relative;
  return true;
}
// The bound depends only on its arguments; provers and verifiers ask for the
// same few codes many times, so results are memoised (thread-safe).
inline bool qa_distance_bound(size_t message_len, size_t index, size_t security_bits, double modulus_log2, double& rel) {
  static std::mutex mu;
  static std::map<std::tuple<size_t, size_t, size_t, double>, std::pair<bool, double>> memo;
  const auto key = std::make_tuple(message_len, index, security_bits, modulus_log2);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = memo.find(key);
    if (it != memo.end()) {
      rel = it->second.second;
      return it->second.first;
    }
  }
  double r = 0.0;
  const bool ok = qa_distance_bound_uncached(message_len, index, security_bits, modulus_log2, r);
  std::lock_guard<std::mutex> g(mu);
  memo[key] = {ok, r};
  rel = r;
  return ok;
}
// brakefold.rs:4-20.
inline size_t queries_for_relative_distance(size_t security_bits, double distance) {
  if (!(std::isfinite(distance) && distance > 0.0 && distance < 1.0)) fail(QF_E_ENCODING, "distance");
  double base = 1.0 - distance / 3.0;
  if (!(base > 0.0 && base < 1.0)) fail(QF_E_ENCODING, "soundness base");
  double q = -double(security_bits) / std::log2(base);
  if (!std::isfinite(q) || q < 0.0) fail(QF_E_ENCODING, "queries");
  return size_t(std::ceil(q));
}
}  // namespace dist

// ---------------------------------------------------------------- QA code
template <class F>
struct QaCode {
  size_t message_len = 0;
  size_t index = 2;
  std::vector<std::vector<F>> alphas;  // alphas[b][row]
  Digest generator_digest{};
  bool systematic_first = false;

  size_t codeword_len() const { return message_len * index; }

  // Encodes one message column into out[0 .. 2*message_len): systematic half
  // then WHT(alpha1 (.) WHT(msg)) (qafold_short.rs:975-1002).
  void encode_into(const F* message, F* out) const {
    if (!(systematic_first && index == 2)) fail(QF_E_ENCODING, "unsupported QA code shape");
    const size_t n = message_len;
    for (size_t i = 0; i < n; ++i) out[i] = message[i];
    F* spec = out + n;
    for (size_t i = 0; i < n; ++i) spec[i] = message[i];
    wht_in_place(spec, n);
    for (size_t i = 0; i < n; ++i) spec[i] = spec[i] * alphas[1][i];
    wht_in_place(spec, n);
  }

  // W(sum_b alpha_b (.) W(left_b)) with the systematic block added directly
  // (qafold_short.rs:1106-1160).
  std::vector<F> generator_left_projection(const std::vector<F>& left) const {
    if (left.size() != codeword_len()) fail(QF_E_ENCODING, "left projection length");
    const size_t n = message_len;
    std::vector<F> projected(n, F::zero()), values(n);
    size_t skip = systematic_first ? 1 : 0;
    for (size_t b = skip; b < index; ++b) {
      for (size_t i = 0; i < n; ++i) values[i] = left[b * n + i];
      wht_in_place(values.data(), n);
      for (size_t i = 0; i < n; ++i) projected[i] += values[i] * alphas[b][i];
    }
    wht_in_place(projected.data(), n);
    if (systematic_first)
      for (size_t i = 0; i < n; ++i) projected[i] += left[i];
    return projected;
  }
  std::vector<F> generator_right_projection(const std::vector<F>& right) const {
    std::vector<F> out(codeword_len());
    encode_into(right.data(), out.data());
    return out;
  }

  size_t num_queries(size_t security_bits, size_t available_rows, double card_log2) const {
    if (available_rows == 0) fail(QF_E_ENCODING, "no rows");
    double rel;
    if (!dist::qa_distance_bound(message_len, index, security_bits, card_log2, rel)) return available_rows;
    // DirectInterleavedV1: zero RF layers, the distance is validated only.
    if (!(std::isfinite(rel) && rel > 0.0 && rel < 1.0)) fail(QF_E_ENCODING, "rf distance");
    if (!(std::isfinite(card_log2) && card_log2 > 1.001)) fail(QF_E_ENCODING, "field log");
    size_t q = dist::queries_for_relative_distance(security_bits, rel);
    return q < available_rows ? q : available_rows;
  }
};

// tensor weights MSB-first: weight(i) = prod_{bit k of i set} point[n-1-k]
// (qafold_short_pc.rs:2826-2855).
template <class F>
std::vector<F> tensor_weights(const std::vector<F>& point) {
  size_t n = point.size();
  std::vector<F> w(size_t(1) << n, F::zero());
  w[0] = F::one();
  size_t filled = 1;
  for (size_t k = n; k-- > 0;) {
    F ch = point[k];
    for (size_t i = 0; i < filled; ++i) w[filled + i] = w[i] * ch;
    filled *= 2;
  }
  return w;
}
template <class F>
F mle_eval_pts(const std::vector<F>& values, const std::vector<F>& point, bool& ok);

template <class F>
F evaluate_generator_mle(const QaCode<F>& code, const std::vector<F>& left_point, const std::vector<F>& right_point) {
  if (left_point.size() != size_t(ilog2(code.codeword_len())) || right_point.size() != size_t(ilog2(code.message_len)))
    fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "generator mle dims");
  // short_tensor_weights: index bit (n-1-k) <-> point[k]; identical to tensor_weights.
  std::vector<F> left = tensor_weights(left_point);
  std::vector<F> right = tensor_weights(right_point);
  std::vector<F> proj = code.generator_right_projection(right);
  F s = F::zero();
  for (size_t i = 0; i < left.size(); ++i) s += left[i] * proj[i];
  return s;
}

inline Digest derive_level_seed(const Digest& seed, size_t level) {
  Blake2s h;
  const char* dom = "qafold-short/qa-level-seed/v1";
  absorb_framed(h, "domain", dom, std::strlen(dom));
  absorb_framed(h, "master-seed", seed.data(), 32);
  absorb_framed_u64(h, "level", level);
  return h.finalize();
}

// The hasher state after the frames shared by every row of one generator
// column (domain, field, modulus, seed, message length, index, block).
template <class F>
Blake2s generator_column_hasher(const Digest& seed, size_t message_len, size_t index, size_t block) {
  Blake2s base;
  const char* dom = "qafold-short/qa-generator-coefficient/v1";
  absorb_framed(base, "domain", dom, std::strlen(dom));
  absorb_framed(base, "field-name", F::kName, std::strlen(F::kName));
  absorb_framed_u64(base, "modulus", F::modulus_u64());
  absorb_framed(base, "seed", seed.data(), 32);
  absorb_framed_u64(base, "message-length", message_len);
  absorb_framed_u64(base, "index", index);
  absorb_framed_u64(base, "block", block);
  return base;
}
// Full-extension fields: UNIFORM_BYTES = 16, two 16-byte lanes per digest
// (qafold_short.rs:2219-2281).  `column` is generator_column_hasher's state.
template <class F>
F sample_generator_element_from(const Blake2s& column, size_t row) {
  Blake2s base = column;
  absorb_framed_u64(base, "row", row);
  for (uint64_t attempt = 0;; ++attempt) {
    Blake2s h = base;
    absorb_framed_u64(h, "attempt", attempt);
    Digest d = h.finalize();
    for (int lane = 0; lane < 2; ++lane) {
      F v;
      if (F::from_uniform_bytes(d.data() + 16 * lane, v)) return v;
    }
  }
}
template <class F>
F sample_generator_element(const Digest& seed, size_t message_len, size_t index, size_t block, size_t row) {
  return sample_generator_element_from<F>(generator_column_hasher<F>(seed, message_len, index, block), row);
}

template <class F>
Digest qa_generator_digest(const std::vector<std::vector<F>>& alphas) {
  Blake2s h;
  const char* dom = "qafold-short/qa-generator/v1";
  absorb_framed(h, "domain", dom, std::strlen(dom));
  absorb_framed(h, "field-name", F::kName, std::strlen(F::kName));
  absorb_framed_u64(h, "modulus", F::modulus_u64());
  absorb_framed_u64(h, "columns", alphas.size());
  absorb_framed_u64(h, "rows", alphas.empty() ? 0 : alphas[0].size());
  // Each coefficient's frame, u64(11) || "coefficient" || u64(16) || bytes,
  // is assembled into a batch that is absorbed in one update.
  static const char kLabel[] = "coefficient";
  constexpr size_t kL = sizeof(kLabel) - 1, kFrame = 8 + kL + 8 + F::kBytes, kBatch = 256;
  std::vector<uint8_t> batch(kFrame * kBatch);
  for (size_t i = 0; i < kBatch; ++i) {
    uint8_t* f = batch.data() + i * kFrame;
    for (int k = 0; k < 8; ++k) f[k] = uint8_t(uint64_t(kL) >> (8 * k));
    std::memcpy(f + 8, kLabel, kL);
    for (int k = 0; k < 8; ++k) f[8 + kL + k] = uint8_t(uint64_t(F::kBytes) >> (8 * k));
  }
  for (size_t col = 0; col < alphas.size(); ++col) {
    absorb_framed_u64(h, "column", col);
    const std::vector<F>& a = alphas[col];
    for (size_t i = 0; i < a.size(); i += kBatch) {
      const size_t n = std::min(kBatch, a.size() - i);
      for (size_t k = 0; k < n; ++k) a[i + k].to_bytes(batch.data() + k * kFrame + 16 + kL);
      h.update(batch.data(), n * kFrame);
    }
  }
  return h.finalize();
}

// ShortQaCode::sample_systematic -> from_group_algebra (qafold_short.rs:699-808).
template <class F>
QaCode<F> sample_systematic(size_t message_len, size_t index, const Digest& seed) {
  if (message_len == 0 || !is_pow2(message_len) || index <= 1 || !is_pow2(index)) fail(QF_E_ENCODING, "qa shape");
  std::vector<std::vector<F>> cols(index, std::vector<F>(message_len, F::zero()));
  cols[0][0] = F::one();
  for (size_t b = 1; b < index; ++b) {
    const Blake2s column = generator_column_hasher<F>(seed, message_len, index, b);
    std::vector<F>& out = cols[b];
#pragma omp parallel for schedule(static) if (message_len >= 4096)
    for (long r = 0; r < long(message_len); ++r) out[size_t(r)] = sample_generator_element_from<F>(column, size_t(r));
  }
  F n_inv = F::from_base(uint32_t(message_len % F::kPrime)).inverse();
  for (auto& a : cols) {
    wht_in_place(a.data(), message_len);
#pragma omp parallel for schedule(static) if (message_len >= 4096)
    for (long r = 0; r < long(message_len); ++r) a[size_t(r)] = a[size_t(r)] * n_inv;
  }
  QaCode<F> code;
  code.message_len = message_len;
  code.index = index;
  code.systematic_first = true;
  for (const F& v : cols[0]) if (v != n_inv) code.systematic_first = false;
  code.generator_digest = qa_generator_digest<F>(cols);
  code.alphas = std::move(cols);
  return code;
}

template <class F>
struct QaSequence {
  size_t witness_size = 0;
  size_t extension_columns = 0;
  size_t switch_ratio = 0;
  size_t rf_layers = 0;
  size_t recursive_index = 2;
  std::vector<QaCode<F>> codes;  // ascending message length
  Digest generator_digest{};
  const QaCode<F>& top() const { return codes.back(); }
};

// ShortQaFold::new_with_recursive_index (qafold_short.rs:1672-1735).
template <class F>
QaSequence<F> build_sequence(size_t witness_size, size_t extension_columns, const Digest& seed) {
  if (witness_size == 0 || !is_pow2(witness_size) || extension_columns <= 1 || !is_pow2(extension_columns))
    fail(QF_E_ENCODING, "sequence shape");
  if (witness_size % extension_columns) fail(QF_E_ENCODING, "sequence divisibility");
  size_t m = witness_size / extension_columns;
  std::vector<size_t> desc;
  for (;;) {
    desc.push_back(m);
    if (m < extension_columns) break;
    if (m % extension_columns) fail(QF_E_ENCODING, "sequence divisibility");
    m /= extension_columns;
  }
  std::vector<size_t> asc(desc.rbegin(), desc.rend());
  QaSequence<F> s;
  s.witness_size = witness_size;
  s.extension_columns = extension_columns;
  s.switch_ratio = extension_columns;
  s.rf_layers = size_t(ilog2(extension_columns));
  s.recursive_index = 2;
  for (size_t level = 0; level < asc.size(); ++level)
    s.codes.push_back(sample_systematic<F>(asc[level], 2, derive_level_seed(seed, level)));
  Blake2s h;
  const char* dom = "qafold-short/qa-sequence-generators/v1";
  absorb_framed(h, "domain", dom, std::strlen(dom));
  absorb_framed_u64(h, "levels", s.codes.size());
  for (size_t level = 0; level < s.codes.size(); ++level) {
    absorb_framed_u64(h, "level", level);
    absorb_framed_u64(h, "message-length", s.codes[level].message_len);
    absorb_framed_u64(h, "index", s.codes[level].index);
    absorb_framed(h, "generator", s.codes[level].generator_digest.data(), 32);
  }
  s.generator_digest = h.finalize();
  return s;
}

}  // namespace qf
