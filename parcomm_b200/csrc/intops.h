// Algorithmic integer operations of the commit kernels, for the integer
// roofline: the thread-level instructions the arithmetic itself needs, per
// unit of work, counted from the operations as the field headers write them
// (f65521_dev.cuh, fkb_dev.cuh, blake2s_dev.cuh).  Address arithmetic, loads,
// stores and shared-memory traffic are not counted: they are what a kernel
// spends beyond the arithmetic, and the gap between these counts and the
// measured instruction rate is what the roofline exposes.
#pragma once
#include <cstdint>

namespace qf_intops {

struct FieldOps {
  double wht_level;   // one WHT level, per element and coefficient
  double mob_level;   // one Mobius level, per element and coefficient
  double reduce;      // reduction of a lazily kept coefficient to canonical form
  double unpack;      // unpack + pack of a stored coefficient
  double mul;         // one extension-field product (element x element)
  int coeffs;         // coefficients per element
};

// F65521^8, lazy butterflies: a WHT pair is one add and one three-operand
// add (a + 2^l p - b), a Mobius pair one three-operand add; a reduction folds
// 2^16 = 15 once (shift, multiply-add) and subtracts p once (subtract,
// minimum); unpack is one extract per coefficient, pack one permute per two.
// The product: 8 multiplies by 17, 64 widening multiply-adds (two issue slots
// each), 8 reductions of about 6 operations.
constexpr FieldOps kF65521{1.0, 0.5, 4.0, 1.5, 8 + 64 * 2 + 8 * 6, 8};
// KoalaBear^4, canonical after every butterfly: addp / subp are an add or
// subtract, the corrected value and an unsigned minimum (3 operations), so a
// WHT pair costs 6 and a Mobius pair 3.  Values stay canonical 32-bit words:
// no reduction and no unpacking.  The product: 3 b_j by two modular additions
// (24), 16 widening products (two slots each), 4 Barrett reductions of about
// 15 operations.
constexpr FieldOps kKoalaBear{3.0, 1.5, 0.0, 0.0, 24 + 16 * 2 + 4 * 15, 4};

// One BLAKE2s compression: 10 rounds of 8 G functions, each 6 additions,
// 4 XORs and 4 rotations.
constexpr double kBlake2sCompression = 10 * 8 * 14;

// A transform pass over n elements: w WHT and m Mobius levels, `reduced`
// canonical stores per element (a fused pass stores twice), `products`
// extension products per element.
inline uint64_t transform_ops(const FieldOps& f, uint64_t n, int w, int m, int reduced, int products) {
  const double per = f.coeffs * (w * f.wht_level + m * f.mob_level + reduced * (f.reduce + f.unpack)) + products * f.mul;
  return uint64_t(per * double(n));
}

// Leaf hashing of `rows` rows of `row_bytes` after a prefix of `prefix`
// bytes, of which the first 64 are absorbed once on the host (midstate).
inline uint64_t leaf_hash_ops(uint64_t rows, uint64_t prefix, uint64_t row_bytes) {
  const uint64_t tail = prefix + row_bytes - 64;
  return uint64_t(double(rows) * double((tail + 63) / 64) * kBlake2sCompression);
}
// Inner nodes: two compressions each (114-byte messages).
inline uint64_t inner_hash_ops(uint64_t nodes) { return uint64_t(double(nodes) * 2 * kBlake2sCompression); }

}  // namespace qf_intops
