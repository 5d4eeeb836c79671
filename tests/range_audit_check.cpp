// The LogUp audit's host side (csrc/host/range_audit.h) on the CPU: the
// table sum through one batched inversion equals the direct sum of
// m_t / (alpha - t) with one inversion per term, for both fields, on random
// and extreme multiplicities (above the base prime, all bins, one bin); and
// alpha is canonical and outside the base field.  Prints one JSON line.
#include <cstdio>
#include <random>
#include <vector>

#include "../parcomm_b200/csrc/host/field65521.h"
#include "../parcomm_b200/csrc/host/fieldkb.h"
#include "../parcomm_b200/csrc/host/range_audit.h"

using namespace qf;

template <class F, class W>
int check_field(std::mt19937_64& rng, int& checked) {
  using T = RangeTable<W>;
  int bad = 0;
  for (int trial = 0; trial < 24; ++trial) {
    uint8_t seed[32];
    for (auto& b : seed) b = uint8_t(rng());
    const F alpha = range_audit_alpha<F>(seed);
    if (in_base_field(alpha)) ++bad;
    std::vector<uint64_t> mult(T::kBins, 0);
    if (trial % 4 == 0) {
      for (auto& m : mult) m = rng() % 5;                   // sparse small counts
    } else if (trial % 4 == 1) {
      mult[rng() % T::kBins] = (uint64_t(1) << 40) + rng() % 1000;  // one bin, count above p
    } else if (trial % 4 == 2) {
      for (auto& m : mult) m = 1;                           // every table value once
    } else {
      for (size_t k = 0; k < T::kBins; k += 1 + rng() % 17) mult[k] = rng() >> 20;  // large counts
    }
    const F fast = logup_table_sum<F, W>(alpha, mult);
    F slow = F::zero();
    for (size_t k = 0; k < T::kBins; ++k)
      if (mult[k]) {
        const F d = alpha - F::from_base(F::small(int(int64_t(k) + T::kMin)));
        slow += d.inverse() * F::from_base(uint32_t(mult[k] % F::modulus_u64()));
      }
    if (!(fast == slow)) ++bad;
    ++checked;
  }
  return bad;
}

int main() {
  std::mt19937_64 rng(20261204);
  int checked = 0;
  const int bad = check_field<Fp8, int8_t>(rng, checked) + check_field<Kb4, int16_t>(rng, checked);
  std::printf("{\"checked\": %d, \"mismatches\": %d}\n", checked, bad);
  return bad ? 1 : 0;
}
