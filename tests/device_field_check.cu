// Host-side check of the device F65521^8 arithmetic (device/f65521_dev.cuh)
// against the host field (host/field65521.h): random and extreme operands.
// Built by tests/test_device_field.py with nvcc and run on the CPU.
#include <cstdio>
#include <cstring>

#include "../parcomm_b200/csrc/device/f65521_dev.cuh"
#include "../parcomm_b200/csrc/host/field65521.h"

static uint64_t state = 0x9e3779b97f4a7c15ull;
static uint64_t next() {
  state ^= state << 13;
  state ^= state >> 7;
  state ^= state << 17;
  return state;
}
static qf::Fp8 sample(int mode) {
  qf::Fp8 v;
  for (int k = 0; k < 8; ++k) {
    uint32_t x = uint32_t(next() % 65521u);
    if (mode == 1) x = 65520u;
    if (mode == 2) x = (next() & 1) ? 65520u : 0u;
    v.c[k] = uint16_t(x);
  }
  return v;
}
static qfd::Fr to_fr(const qf::Fp8& v) {
  qfd::Fr r;
  for (int k = 0; k < 8; ++k) r.c[k] = v.c[k];
  return r;
}
static bool same(const qfd::Fr& a, const qf::Fp8& b) {
  for (int k = 0; k < 8; ++k)
    if (a.c[k] != b.c[k]) return false;
  return true;
}

int main() {
  long bad = 0, n = 0;
  for (int it = 0; it < 300000; ++it) {
    const int mode = it < 1000 ? 1 : (it < 5000 ? 2 : 0);
    const qf::Fp8 a = sample(mode), b = sample(mode);
    const qfd::Fr fa = to_fr(a), fb = to_fr(b);
    bad += !same(qfd::mul(fa, fb), a * b);
    bad += !same(qfd::add(fa, fb), a + b);
    bad += !same(qfd::sub(fa, fb), a - b);
    const uint32_t s = uint32_t(next() % 65521u);
    bad += !same(qfd::mul_base(fa, s), a * qf::Fp8::from_base(s));
    const uint64_t v = next() & ((uint64_t(1) << 40) - 1);
    bad += qfd::red40(v) != uint32_t(v % 65521u);
    const uint32_t w = uint32_t(next());
    bad += qfd::red32(w) != w % 65521u;
    n += 6;
  }
  // Signed sums below 2^62 in magnitude.
  for (int it = 0; it < 200000; ++it) {
    int64_t v = int64_t(next() >> 2) * ((next() & 1) ? 1 : -1);
    if (it < 4) v = (it & 1 ? -1 : 1) * ((int64_t(1) << 62) - 1 - it / 2);
    int64_t want = v % int64_t(65521);
    if (want < 0) want += 65521;
    bad += qfd::red_signed(v) != uint32_t(want);
    ++n;
  }
  // Lazy sums of products: short random runs, and 2^20 products of all-(p-1)
  // operands (the largest raw coefficient growth) reduced once.
  for (int run = 0; run < 2000; ++run) {
    const int len = run < 1999 ? 1 + int(next() % 64) : (1 << 20);
    const int mode = run == 1999 ? 1 : (run < 200 ? 2 : 0);
    qfd::Acc acc = qfd::acc_zero();
    qf::Fp8 want = qf::Fp8::zero();
    for (int i = 0; i < len; ++i) {
      const qf::Fp8 a = sample(mode), b = sample(mode);
      qfd::mul_acc(acc, to_fr(a), to_fr(b));
      want += a * b;
    }
    bad += !same(qfd::acc_reduce(acc), want);
    ++n;
  }
  std::printf("{\"checked\": %ld, \"mismatches\": %ld}\n", n, bad);
  return bad != 0;
}
