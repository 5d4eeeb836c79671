// LogUp range audit of BVA values over the 8- or 16-bit table.
//
// A separate check beside the proof, never part of it: nothing here enters a
// transcript or the proof bytes.  For the values v_i of a committed BVA
// (int8 entries lifted into F65521, int16 payloads into KoalaBear, as
// field.rs:24-29 lifts them) and the table T of every value of the entry type,
// the LogUp identity
//
//     sum_i 1 / (alpha - v_i)  ==  sum_{t in T} m_t / (alpha - t)
//
// holds for a random alpha of the extension field exactly when the multiset
// {v_i} is the multiset with multiplicities m_t over T (up to a soundness
// error of about |{v_i}| / |F^d|).  The left side is accumulated per value on
// the device without looking at the multiplicities; the right side comes from
// them.
//
// alpha is drawn from a 32-byte seed by BLAKE2s with this library's own
// domain, rejecting non-canonical draws and draws in the base field (those
// could equal a table value).
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>

#include "blake2s.h"

namespace qf {

constexpr const char* kRangeAuditDomain = "parcomm-b200/logup-range-audit/v1";

// Table of the entry type W: the values min, min + 1, ..., max; bin k holds
// the value k + min.
template <class W>
struct RangeTable {
  static constexpr int64_t kMin = sizeof(W) == 1 ? -128 : -32768;
  static constexpr size_t kBins = sizeof(W) == 1 ? 256 : 65536;
};

template <class F>
bool in_base_field(const F& a) {
  for (int i = 1; i < int(sizeof(a.c) / sizeof(a.c[0])); ++i)
    if (a.c[i] != 0) return false;
  return true;
}

// alpha = the first accepted draw of BLAKE2s(frame(domain) || frame(field) ||
// frame(seed) || frame(counter)), counter = 0, 1, ...
template <class F>
F range_audit_alpha(const uint8_t seed[32]) {
  for (uint64_t counter = 0;; ++counter) {
    Blake2s h;
    absorb_framed(h, "domain", kRangeAuditDomain, std::strlen(kRangeAuditDomain));
    absorb_framed(h, "field", F::kName, std::strlen(F::kName));
    absorb_framed(h, "seed", seed, 32);
    absorb_framed_u64(h, "counter", counter);
    const Digest d = h.finalize();
    F a;
    if (F::from_uniform_bytes(d.data(), a) && !in_base_field(a)) return a;
  }
}

// sum_t m_t / (alpha - t) over the nonzero multiplicities, with one field
// inversion (prefix products, Montgomery's batch inversion).
template <class F, class W>
F logup_table_sum(const F& alpha, const std::vector<uint64_t>& mult) {
  using T = RangeTable<W>;
  std::vector<F> den;
  std::vector<uint64_t> count;
  for (size_t k = 0; k < mult.size() && k < T::kBins; ++k)
    if (mult[k]) {
      den.push_back(alpha - F::from_base(F::small(int(int64_t(k) + T::kMin))));
      count.push_back(mult[k]);
    }
  if (den.empty()) return F::zero();
  std::vector<F> prefix(den.size());
  F acc = F::one();
  for (size_t i = 0; i < den.size(); ++i) { prefix[i] = acc; acc = acc * den[i]; }
  F inv = acc.inverse();  // nonzero: alpha is outside the base field
  F sum = F::zero();
  for (size_t i = den.size(); i-- > 0;) {
    const F inv_i = inv * prefix[i];
    inv = inv * den[i];
    sum += inv_i * F::from_base(uint32_t(count[i] % F::modulus_u64()));
  }
  return sum;
}

}  // namespace qf
