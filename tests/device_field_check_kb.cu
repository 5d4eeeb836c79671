// Host-side check of the device KoalaBear^4 arithmetic (device/fkb_dev.cuh)
// against the host field (host/fieldkb.h): random and extreme operands, the
// Barrett reduction over the whole u64 range, the transform butterflies and
// the conversion of packed signed 16-bit payloads.  Built by
// tests/test_device_field.py with nvcc and run on the CPU.
#include <cstdio>
#include <cstring>

#include "../parcomm_b200/csrc/device/fkb_dev.cuh"
#include "../parcomm_b200/csrc/host/fieldkb.h"

static uint64_t state = 0x2545f4914f6cdd1dull;
static uint64_t next() {
  state ^= state << 13;
  state ^= state >> 7;
  state ^= state << 17;
  return state;
}
static const uint32_t P = qf::PKB;
static qf::Kb4 sample(int mode) {
  qf::Kb4 v;
  for (int k = 0; k < 4; ++k) {
    uint32_t x = uint32_t(next() % P);
    if (mode == 1) x = P - 1;
    if (mode == 2) x = (next() & 1) ? P - 1 : 0u;
    v.c[k] = x;
  }
  return v;
}
static qfdkb::Fr to_fr(const qf::Kb4& v) {
  qfdkb::Fr r;
  for (int k = 0; k < 4; ++k) r.c[k] = v.c[k];
  return r;
}
static bool same(const qfdkb::Fr& a, const qf::Kb4& b) {
  for (int k = 0; k < 4; ++k)
    if (a.c[k] != b.c[k]) return false;
  return true;
}

int main() {
  long bad = 0, n = 0;
  for (int it = 0; it < 300000; ++it) {
    const int mode = it < 1000 ? 1 : (it < 5000 ? 2 : 0);
    const qf::Kb4 a = sample(mode), b = sample(mode);
    const qfdkb::Fr fa = to_fr(a), fb = to_fr(b);
    bad += !same(qfdkb::mul(fa, fb), a * b);
    bad += !same(qfdkb::add(fa, fb), a + b);
    bad += !same(qfdkb::sub(fa, fb), a - b);
    const uint32_t s = uint32_t(next() % P);
    bad += !same(qfdkb::mul_base(fa, s), a.mul_prime(s));
    uint64_t v = next();
    if (it < 64) v = ~uint64_t(0) - uint64_t(it);  // the top of the range
    bad += qfdkb::red64(v) != uint32_t(v % P);
    // Butterflies on canonical values.
    uint32_t lo = fa.c[0], hi = fb.c[0];
    qfdkb::bfly_wht(lo, hi, qfdkb::tile_bound(0));
    bad += lo != qf::kb_add(a.c[0], b.c[0]) || hi != qf::kb_sub(a.c[0], b.c[0]);
    uint32_t h2 = fb.c[1];
    qfdkb::bfly_mobius(fa.c[1], h2, qfdkb::tile_bound(0));
    bad += h2 != qf::kb_sub(b.c[1], a.c[1]);
    // Four packed signed 16-bit payloads.
    const uint2 raw = make_uint2(uint32_t(next()), uint32_t(next()));
    const qfdkb::Fr w = qfdkb::weights_to_fr(raw);
    const int16_t e[4] = {int16_t(raw.x & 0xffff), int16_t(raw.x >> 16), int16_t(raw.y & 0xffff), int16_t(raw.y >> 16)};
    for (int k = 0; k < 4; ++k) bad += w.c[k] != qf::Kb4::small(e[k]);
    n += 11;
  }
  for (int it = 0; it < 200000; ++it) {
    int64_t v = int64_t(next() >> 2) * ((next() & 1) ? 1 : -1);
    if (it < 4) v = (it & 1 ? -1 : 1) * ((int64_t(1) << 62) - 1 - it / 2);
    int64_t want = v % int64_t(P);
    if (want < 0) want += P;
    bad += qfdkb::red_signed(v) != uint32_t(want);
    ++n;
  }
  for (int run = 0; run < 500; ++run) {
    const int len = 1 + int(next() % 64);
    qfdkb::Acc acc = qfdkb::acc_zero();
    qf::Kb4 want = qf::Kb4::zero();
    for (int i = 0; i < len; ++i) {
      const qf::Kb4 a = sample(run < 50 ? 1 : 0), b = sample(run < 50 ? 1 : 0);
      qfdkb::mul_acc(acc, to_fr(a), to_fr(b));
      want += a * b;
    }
    bad += !same(qfdkb::acc_reduce(acc), want);
    ++n;
  }
  std::printf("{\"checked\": %ld, \"mismatches\": %ld}\n", n, bad);
  return bad != 0;
}
