// ORACLE (test infrastructure only): C entry points over the CPU restatement
// in cpu_backend.h, used by tests/, __graft_entry__.smoke() and the bench's
// CPU-baseline leg to compare results with.  Never linked into the product library.
//
// Pinned by the reference's own golden vectors:
//   * demo proof (qafold/f65521/src/main.rs:108-145, validation/qafold8-smoke-final/run.log)
//   * native opening + Decide wire fixture (qafold_short_pc.rs:3605-3647)
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <cstdlib>
#include <string>

#include "cpu_backend.h"
#include "cpu_shard.h"
#include "../parcomm_b200/csrc/host/range_audit.h"

using namespace qf;
using F = Fp8;

namespace {
thread_local std::string g_err;
template <class Fn>
int guarded(Fn&& fn) {
  try {
    fn();
    return 0;
  } catch (const QfError& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -7;
  }
}
uint8_t* dup(const std::vector<uint8_t>& v) {
  uint8_t* p = static_cast<uint8_t*>(std::malloc(v.size() ? v.size() : 1));
  if (!v.empty()) std::memcpy(p, v.data(), v.size());
  return p;
}
template <class G = F>
G sample_uniform(StdRng& rng) {
  for (;;) {
    uint8_t b[16];
    uint64_t a = rng.next_u64(), c = rng.next_u64();
    for (int i = 0; i < 8; ++i) { b[i] = uint8_t(a >> (8 * i)); b[8 + i] = uint8_t(c >> (8 * i)); }
    G v;
    if (G::from_uniform_bytes(b, v)) return v;
  }
}
std::vector<Shape> shapes_of(const uint64_t* s, size_t n) {
  std::vector<Shape> out;
  for (size_t i = 0; i < n; ++i) out.push_back({size_t(s[2 * i]), size_t(s[2 * i + 1])});
  return out;
}
// LogUp range audit, from the definitions: m_t counts the values equal to t;
// lhs = sum over the values of (alpha - v)^-1, each distinct value's inverse
// computed once; rhs = sum_t m_t (alpha - t)^-1 with one inversion per term.
// alpha comes from the same seed derivation as the library's.
template <class G, class T>
int range_audit_impl(const T* values, uint64_t n, const uint8_t seed[32], uint64_t* mult_out, uint8_t alpha_out[16],
                     uint8_t lhs_out[16], uint8_t rhs_out[16]) {
  return guarded([&] {
    using Tab = RangeTable<T>;
    const G alpha = range_audit_alpha<G>(seed);
    std::vector<uint64_t> mult(Tab::kBins, 0);
    std::vector<G> inv(Tab::kBins);
    std::vector<bool> have(Tab::kBins, false);
    G lhs = G::zero();
    for (uint64_t i = 0; i < n; ++i) {
      const size_t k = size_t(int64_t(values[i]) - Tab::kMin);
      ++mult[k];
      if (!have[k]) {
        inv[k] = (alpha - G::from_base(G::small(int(values[i])))).inverse();
        have[k] = true;
      }
      lhs += inv[k];
    }
    G rhs = G::zero();
    for (size_t k = 0; k < Tab::kBins; ++k)
      if (mult[k]) {
        const G d = alpha - G::from_base(G::small(int(int64_t(k) + Tab::kMin)));
        rhs += d.inverse() * G::from_base(uint32_t(mult[k] % G::modulus_u64()));
      }
    std::memcpy(mult_out, mult.data(), mult.size() * 8);
    alpha.to_bytes(alpha_out);
    lhs.to_bytes(lhs_out);
    rhs.to_bytes(rhs_out);
  });
}
template <class G, class T>
int prove_impl(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
               const T* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, uint8_t** roots,
               size_t* roots_len, uint8_t** claims_out, size_t* claims_out_len, uint8_t** proof, size_t* proof_len,
               double* times_ms) {
  return guarded([&] {
    Config c;
    c.chunk_log = chunk_log;
    c.packed_log = packed_log;
    c.query_rf_bits = rf_bits;
    auto P = make_parameters<G>(shapes_of(shapes, n_shapes), c);
    std::vector<Claim<G>> given;
    if (claims_in) {
      ByteReader r(claims_in, claims_len);
      for (const Shape& s : P->layout.shapes) {
        Claim<G> cl;
        for (int i = 0; i < ilog2(next_pow2(s.rows)); ++i) cl.row.push_back(r.field<G>());
        for (int i = 0; i < ilog2(next_pow2(s.cols)); ++i) cl.col.push_back(r.field<G>());
        cl.value = r.field<G>();
        given.push_back(cl);
      }
    }
    auto res = qf_oracle::prove_all<G, T>(*P, bva, n_values, claims_in == nullptr, claims_in ? &given : nullptr);
    ByteWriter rw, cw;
    for (const auto& d : res.statement.roots) rw.digest(d);
    for (const auto& cl : res.claims) {
      for (const G& v : cl.row) cw.field(v);
      for (const G& v : cl.col) cw.field(v);
      cw.field(cl.value);
    }
    *roots = dup(rw.out);
    *roots_len = rw.out.size();
    *claims_out = dup(cw.out);
    *claims_out_len = cw.out.size();
    *proof = dup(res.wire);
    *proof_len = res.wire.size();
    if (times_ms) { times_ms[0] = res.commit_ms; times_ms[1] = res.open_ms; }
  });
}

template <class G, class T>
int commit_roots_impl(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                      const T* bva, uint64_t n_values, uint8_t* roots_out, size_t cap) {
  return guarded([&] {
    Config c;
    c.chunk_log = chunk_log;
    c.packed_log = packed_log;
    c.query_rf_bits = rf_bits;
    auto P = make_parameters<G>(shapes_of(shapes, n_shapes), c);
    validate_values(P->layout, bva, n_values);
    if (cap < 32 * P->blocks()) fail(-9, "roots buffer too small");
    qf_oracle::CpuBackend<G, T> be(*P, bva, n_values);
    for (size_t b = 0; b < P->blocks(); ++b) {
      Digest d = be.commit_block(b);
      std::memcpy(roots_out + 32 * b, d.data(), 32);
    }
  });
}

// The demo bundle (main.rs:108-145): shapes 31x37, 65x17, 1x7, 9x1, entry
// (e * 73 + i * 19) truncated to the payload width, chunk 10, packed_log 4.
template <class G, class T, class U>
int demo_impl(uint8_t digest_out[32], uint64_t* proof_len, uint64_t* statement_json_len) {
  return guarded([&] {
    std::vector<Shape> shapes = {{31, 37}, {65, 17}, {1, 7}, {9, 1}};
    Config c;
    c.chunk_log = 10;
    c.packed_log = 4;
    auto P = make_parameters<G>(shapes, c);
    std::vector<std::vector<T>> mats;
    for (size_t i = 0; i < shapes.size(); ++i) {
      std::vector<T> m(shapes[i].rows * shapes[i].cols);
      for (size_t e = 0; e < m.size(); ++e) m[e] = T(U(e * 73 + i * 19));
      mats.push_back(m);
    }
    auto vals = layout_encode<T>(P->layout, mats);
    auto res = qf_oracle::prove_all<G, T>(*P, vals.data(), vals.size(), true);
    Digest d = blake2s(res.wire.data(), res.wire.size());
    std::memcpy(digest_out, d.data(), 32);
    *proof_len = res.wire.size();
    *statement_json_len = commitment_json(res.statement).size();
  });
}

template <class G>
int verify_impl(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                const uint8_t* roots, const uint8_t* claims_in, size_t claims_len, const uint8_t* proof, size_t proof_len) {
  return guarded([&] {
    Config c;
    c.chunk_log = chunk_log;
    c.packed_log = packed_log;
    c.query_rf_bits = rf_bits;
    auto P = make_parameters<G>(shapes_of(shapes, n_shapes), c);
    std::vector<Digest> rs(P->blocks());
    for (size_t b = 0; b < rs.size(); ++b) std::memcpy(rs[b].data(), roots + 32 * b, 32);
    ByteReader r(claims_in, claims_len);
    std::vector<Claim<G>> cl;
    for (const Shape& s : P->layout.shapes) {
      Claim<G> x;
      for (int i = 0; i < ilog2(next_pow2(s.rows)); ++i) x.row.push_back(r.field<G>());
      for (int i = 0; i < ilog2(next_pow2(s.cols)); ++i) x.col.push_back(r.field<G>());
      x.value = r.field<G>();
      cl.push_back(x);
    }
    verify_proof(*P, make_statement(*P, rs), cl, proof_from_bytes<G>(proof, proof_len));
  });
}
// One rank of a block-sharded proof (csrc/host/sharded.h) with the CPU shard
// standing in for its device.  Every rank passes the whole BVA; the shard
// keeps only its own blocks.  `claims` may be null: each rank then takes its
// part of the benchmark claims and the parts are summed.
template <class G, class T>
int prove_sharded_impl(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                       const T* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, int rank, int world,
                       CallbackComm::Fn gather, CallbackComm::ReduceFn reduce, void* comm_ctx, uint8_t** roots,
                       size_t* roots_len, uint8_t** claims_out, size_t* claims_out_len, uint8_t** proof,
                       size_t* proof_len) {
  return guarded([&] {
    Config c;
    c.chunk_log = chunk_log;
    c.packed_log = packed_log;
    c.query_rf_bits = rf_bits;
    auto P = make_parameters<G>(shapes_of(shapes, n_shapes), c);
    validate_values(P->layout, bva, n_values);
    CallbackComm comm(rank, world, gather, comm_ctx, reduce);
    BlockShards shards(P->blocks(), world);
    qf_oracle::CpuShard<G, T> shard(*P, bva, n_values, shards, rank);
    ShardedBackend<G> be(*P, shard, comm);
    std::vector<Digest> rs = be.commit_all();
    std::vector<Claim<G>> cl;
    if (claims_in) {
      ByteReader r(claims_in, claims_len);
      for (const Shape& s : P->layout.shapes) {
        Claim<G> x;
        for (int i = 0; i < ilog2(next_pow2(s.rows)); ++i) x.row.push_back(r.field<G>());
        for (int i = 0; i < ilog2(next_pow2(s.cols)); ++i) x.col.push_back(r.field<G>());
        x.value = r.field<G>();
        cl.push_back(x);
      }
    } else {
      cl = sum_claims(comm, qf_oracle::evaluate_claims(*P, shard.masked.data(), n_values,
                                                       benchmark_points<G>(make_statement(*P, rs))));
    }
    std::vector<uint8_t> wire = prove_sharded(*P, be, rs, cl);
    ByteWriter rw, cw;
    for (const auto& d : rs) rw.digest(d);
    for (const auto& x : cl) {
      for (const G& v : x.row) cw.field(v);
      for (const G& v : x.col) cw.field(v);
      cw.field(x.value);
    }
    *roots = dup(rw.out);
    *roots_len = rw.out.size();
    *claims_out = dup(cw.out);
    *claims_out_len = cw.out.size();
    *proof = dup(wire);
    *proof_len = wire.size();
  });
}
// The compiled query of `claims` (tbv::compile from a fresh transcript) in
// dense form, for a check against its definition: one blob of
//   dense weights (logical x 16 B) || query claim || the point of log2(logical)
//   "evaluation" challenges drawn next || Query::evaluation at it ||
//   cross terms at `stride`: positive (stride - 1) || negative (stride - 1).
template <class G, class T>
int tbv_dense_impl(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                   const T* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, uint32_t stride,
                   uint8_t** out, size_t* out_len) {
  return guarded([&] {
    Config c;
    c.chunk_log = chunk_log;
    c.packed_log = packed_log;
    c.query_rf_bits = rf_bits;
    auto P = make_parameters<G>(shapes_of(shapes, n_shapes), c);
    validate_values(P->layout, bva, n_values);
    if (stride < 2 || !is_pow2(stride)) fail(-9, "stride");
    ByteReader r(claims_in, claims_len);
    std::vector<Claim<G>> cl;
    for (const Shape& s : P->layout.shapes) {
      Claim<G> x;
      for (int i = 0; i < ilog2(next_pow2(s.rows)); ++i) x.row.push_back(r.field<G>());
      for (int i = 0; i < ilog2(next_pow2(s.cols)); ++i) x.col.push_back(r.field<G>());
      x.value = r.field<G>();
      cl.push_back(x);
    }
    Transcript<G> t;
    Query<G> q = compile(P->layout, cl, t);
    std::vector<G> dense(P->layout.logical, G::zero());
    for (const Term<G>& term : q.terms)
      for (size_t i = 0; i < term.len(); ++i) dense[term.offset + i] += term.weight(i);
    std::vector<G> point;
    for (int i = 0; i < ilog2(P->layout.logical); ++i) point.push_back(t.challenge("evaluation"));
    qf_oracle::CpuBackend<G, T> be(*P, bva, n_values);
    std::vector<G> pos, neg;
    be.cross_terms(q, stride, pos, neg);
    ByteWriter w;
    for (const G& v : dense) w.field(v);
    w.field(q.claim);
    for (const G& v : point) w.field(v);
    w.field(q.evaluation(point));
    for (const G& v : pos) w.field(v);
    for (const G& v : neg) w.field(v);
    *out = dup(w.out);
    *out_len = w.out.size();
  });
}
// Element-wise a * b, a^-1 (0 for a = 0) and a^p (one Frobenius step) of n
// canonical 16-byte elements each, for checks against the definitions.
template <class G>
int field_ops_impl(const uint8_t* a, const uint8_t* b, size_t n, uint8_t* prod, uint8_t* inv, uint8_t* frob) {
  return guarded([&] {
    for (size_t i = 0; i < n; ++i) {
      G x, y;
      if (!G::from_bytes(a + 16 * i, x) || !G::from_bytes(b + 16 * i, y)) fail(-9, "non-canonical element");
      (x * y).to_bytes(prod + 16 * i);
      (x.is_zero() ? G::zero() : x.inverse()).to_bytes(inv + 16 * i);
      x.frobenius(1).to_bytes(frob + 16 * i);
    }
  });
}
// The single-block packed PCS (PackedPcs::{new, commit, open, verify},
// packed.rs:132-484) over a table of 2^log_n base-field values given as
// canonical integers: commit, open at `point` (log_n elements) under `ctx`;
// outputs the root, the claimed value and the opening's bytes.
template <class G>
int packed_open_impl(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], const int32_t* values,
                     const uint8_t* point, const uint8_t* ctx, size_t ctx_len, uint8_t root[32], uint8_t value[16],
                     uint8_t** proof, size_t* proof_len) {
  return guarded([&] {
    std::array<uint8_t, 32> sd;
    std::memcpy(sd.data(), seed, 32);
    Parameters<G> P;
    P.pcs = PackedPcs<G>::create(log_n, columns, bits, sd);
    P.block_len = size_t(1) << log_n;
    for (size_t i = 0; i < P.block_len; ++i)
      if (values[i] < 0 || uint64_t(values[i]) >= G::modulus_u64()) fail(-9, "non-canonical base value");
    qf_oracle::CpuBackend<G, int32_t> be(P, values, P.block_len);
    const Digest d = be.commit();
    std::vector<G> pt;
    ByteReader r(point, 16 * size_t(log_n));
    for (uint32_t i = 0; i < log_n; ++i) pt.push_back(r.field<G>());
    BatchOpening<G> op = open_single(P.pcs, be, d, pt, std::vector<uint8_t>(ctx, ctx + ctx_len));
    std::memcpy(root, d.data(), 32);
    op.claimed_value.to_bytes(value);
    *proof = dup(op.wire);
    *proof_len = op.wire.size();
  });
}
template <class G>
int packed_verify_impl(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], const uint8_t root[32],
                       const uint8_t* point, const uint8_t value[16], const uint8_t* proof, size_t proof_len,
                       const uint8_t* ctx, size_t ctx_len) {
  return guarded([&] {
    std::array<uint8_t, 32> sd;
    std::memcpy(sd.data(), seed, 32);
    PackedPcs<G> pcs = PackedPcs<G>::create(log_n, columns, bits, sd);
    Digest d;
    std::memcpy(d.data(), root, 32);
    std::vector<G> pt;
    ByteReader r(point, 16 * size_t(log_n));
    for (uint32_t i = 0; i < log_n; ++i) pt.push_back(r.field<G>());
    ByteReader rv(value, 16);
    const G v = rv.field<G>();
    if (!verify_single(pcs, d, pt, v, proof, proof_len, std::vector<uint8_t>(ctx, ctx + ctx_len)))
      fail(QF_E_INVALID_COMMITMENT, "packed opening rejected");
  });
}
// The batched packed PCS (open_batch_impl, packed_batch.rs:139-319) over
// `blocks` tables of 2^log_n canonical base values each: every block
// committed, then one opening at `point` (log_n + log2(blocks) elements, the
// block coordinates first).  Outputs the blocks' roots, the claimed value
// and the opening's bytes.
template <class G>
int packed_open_batch_impl(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], uint32_t blocks,
                           const int32_t* values, const uint8_t* point, const uint8_t* ctx, size_t ctx_len,
                           uint8_t* roots, uint8_t value[16], uint8_t** proof, size_t* proof_len) {
  return guarded([&] {
    if (blocks < 2 || !is_pow2(blocks)) fail(-9, "blocks");
    std::array<uint8_t, 32> sd;
    std::memcpy(sd.data(), seed, 32);
    Parameters<G> P;
    P.pcs = PackedPcs<G>::create(log_n, columns, bits, sd);
    P.block_len = size_t(1) << log_n;
    const size_t n = P.block_len * blocks;
    for (size_t i = 0; i < n; ++i)
      if (values[i] < 0 || uint64_t(values[i]) >= G::modulus_u64()) fail(-9, "non-canonical base value");
    qf_oracle::CpuBackend<G, int32_t> be(P, values, n);
    std::vector<Digest> rs;
    for (uint32_t b = 0; b < blocks; ++b) rs.push_back(be.commit_block(b));
    const size_t k = log_n + ilog2(blocks);
    std::vector<G> pt;
    ByteReader r(point, 16 * k);
    for (size_t i = 0; i < k; ++i) pt.push_back(r.field<G>());
    BatchOpening<G> op = open_batch(P.pcs, be, rs, pt, std::vector<uint8_t>(ctx, ctx + ctx_len));
    for (uint32_t b = 0; b < blocks; ++b) std::memcpy(roots + 32 * b, rs[b].data(), 32);
    op.claimed_value.to_bytes(value);
    *proof = dup(op.wire);
    *proof_len = op.wire.size();
  });
}
template <class G>
int packed_verify_batch_impl(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], uint32_t blocks,
                             const uint8_t* roots, const uint8_t* point, uint32_t point_len, const uint8_t value[16],
                             const uint8_t* proof, size_t proof_len, const uint8_t* ctx, size_t ctx_len) {
  return guarded([&] {
    std::array<uint8_t, 32> sd;
    std::memcpy(sd.data(), seed, 32);
    PackedPcs<G> pcs = PackedPcs<G>::create(log_n, columns, bits, sd);
    std::vector<Digest> rs(blocks);
    for (uint32_t b = 0; b < blocks; ++b) std::memcpy(rs[b].data(), roots + 32 * b, 32);
    std::vector<G> pt;
    ByteReader r(point, 16 * size_t(point_len));
    for (uint32_t i = 0; i < point_len; ++i) pt.push_back(r.field<G>());
    ByteReader rv(value, 16);
    const G v = rv.field<G>();
    if (!verify_batch(pcs, rs, pt, v, proof, proof_len, std::vector<uint8_t>(ctx, ctx + ctx_len)))
      fail(QF_E_INVALID_COMMITMENT, "batch opening rejected");
  });
}
// The codeword-fold binding (prove/verify_codeword_fold,
// qafold_short_batch.rs:77-240): the blocks are folded with the base weights
// `fold_w`, the folded codeword committed, and the binding rows sampled by
// `seed` written; the verifier then checks them against the block roots
// under the weights `check_w`.  `accepted` <- the verifier's answer.
template <class G>
int codeword_fold_impl(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t pcs_seed[32], uint32_t blocks,
                       const int32_t* values, const uint32_t* fold_w, const uint8_t seed[32], const uint32_t* check_w,
                       int* accepted) {
  return guarded([&] {
    if (blocks < 2 || !is_pow2(blocks)) fail(-9, "blocks");
    std::array<uint8_t, 32> sd;
    std::memcpy(sd.data(), pcs_seed, 32);
    Parameters<G> P;
    P.pcs = PackedPcs<G>::create(log_n, columns, bits, sd);
    P.block_len = size_t(1) << log_n;
    qf_oracle::CpuBackend<G, int32_t> be(P, values, P.block_len * blocks);
    std::vector<Digest> rs;
    for (uint32_t b = 0; b < blocks; ++b) rs.push_back(be.commit_block(b));
    std::vector<G> fw, cw;
    for (uint32_t b = 0; b < blocks; ++b) {
      fw.push_back(G::from_base(fold_w[b] % uint32_t(G::modulus_u64())));
      cw.push_back(G::from_base(check_w[b] % uint32_t(G::modulus_u64())));
    }
    const Digest folded = be.fold_and_commit(fw);
    Digest s;
    std::memcpy(s.data(), seed, 32);
    const auto& pp = *P.pcs.pp;
    RowSelection sel = make_selection(pp.num_queries(pp.levels() - 1, pp.top_ext_rows()), pp.top_ext_rows(), s);
    const std::vector<uint8_t> binding = be.binding_rows(sel, rs);
    *accepted = verify_codeword_fold(pp, rs, cw, folded, s, binding.data(), binding.size()) ? 1 : 0;
  });
}
// The prover without the layout check of the weights (the reference's
// commit_unchecked, protocol.rs:333-369): `n_values` entries (up to the
// logical length, so the implicit zero suffix can be overwritten) are
// committed as given and proved against the given claims.  A nonzero entry
// in a bucket's padding or in the suffix must make the proof fail.
template <class G, class T>
int prove_unchecked_impl(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log,
                         uint32_t rf_bits, const T* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len,
                         uint8_t** proof, size_t* proof_len) {
  return guarded([&] {
    Config c;
    c.chunk_log = chunk_log;
    c.packed_log = packed_log;
    c.query_rf_bits = rf_bits;
    auto P = make_parameters<G>(shapes_of(shapes, n_shapes), c);
    if (n_values > P->layout.logical) fail(-9, "more values than the logical length");
    ByteReader r(claims_in, claims_len);
    std::vector<Claim<G>> cl;
    for (const Shape& s : P->layout.shapes) {
      Claim<G> x;
      for (int i = 0; i < ilog2(next_pow2(s.rows)); ++i) x.row.push_back(r.field<G>());
      for (int i = 0; i < ilog2(next_pow2(s.cols)); ++i) x.col.push_back(r.field<G>());
      x.value = r.field<G>();
      cl.push_back(x);
    }
    qf_oracle::CpuBackend<G, T> be(*P, bva, n_values);
    std::vector<Digest> rs;
    for (size_t b = 0; b < P->blocks(); ++b) rs.push_back(be.commit_block(b));
    Transcript<G> t = statement_transcript(*P, make_statement(*P, rs), cl);
    Query<G> q = compile(P->layout, cl, t);
    auto [eo, term] = eo_prove<G>(be, P->layout.logical, size_t(1) << P->config.packed_log, q, t);
    std::vector<uint8_t> ctx = opening_context<G>(t.state, 0);
    BatchOpening<G> op = rs.size() > 1 ? open_batch(P->pcs, be, rs, term.point_msb, ctx)
                                       : open_single(P->pcs, be, rs[0], term.point_msb, ctx);
    check(op.claimed_value * term.scale == term.value, "QAFold/EO terminal mismatch");
    Proof<G> pr;
    pr.eo = eo;
    pr.opening_value = op.claimed_value;
    pr.opening_proof = std::move(op.wire);
    const std::vector<uint8_t> wire = proof_to_bytes(pr);
    *proof = dup(wire);
    *proof_len = wire.size();
  });
}
// The code sequence of a packed PCS over 2^log_n base values with
// `columns` extension columns at `bits` of security: per level (ascending
// message length) the message length, the index, the codeword length and the
// query counts num_queries(level, available) with the codeword's rows
// available and with no limit.  `card_log2` <- log2 of the field's size.
template <class G>
int query_counts_impl(uint32_t log_n, uint32_t columns, uint32_t bits, uint64_t* rows, size_t cap, size_t* levels,
                      double* card_log2) {
  return guarded([&] {
    const size_t n_witness = size_t(1) << (log_n - ilog2(G::kLanes));
    Digest seed;
    seed.fill(0x51);
    PcsParams<G> pp;
    pp.card_log2 = cardinality_log2<G>();
    pp.security_bits = bits;
    pp.extension_columns = columns;
    pp.seq = build_sequence<G>(n_witness, columns, seed);
    *levels = pp.levels();
    *card_log2 = pp.card_log2;
    if (cap < 5 * pp.levels()) fail(-9, "output buffer too small");
    for (size_t l = 0; l < pp.levels(); ++l) {
      const QaCode<G>& c = pp.seq.codes[l];
      rows[5 * l + 0] = c.message_len;
      rows[5 * l + 1] = c.index;
      rows[5 * l + 2] = c.codeword_len();
      rows[5 * l + 3] = pp.num_queries(l, c.codeword_len());
      rows[5 * l + 4] = pp.num_queries(l, SIZE_MAX);
    }
  });
}
// Ranks as threads of one process, for the sharding layer's tests at world
// sizes that would be slow as processes: an all-gather through shared slots
// between two barriers.  A rank that fails marks the group, so the others
// stop at their next barrier instead of waiting; every wait is bounded.
struct ThreadGroup {
  explicit ThreadGroup(int n) : n(n), slots(size_t(n)) {}
  const int n;
  std::mutex mu;
  std::condition_variable cv;
  int arrived = 0;
  uint64_t generation = 0;
  bool aborted = false;
  std::vector<std::vector<uint8_t>> slots;
  void barrier() {
    std::unique_lock<std::mutex> lk(mu);
    if (aborted) fail(QF_E_PROTOCOL, "another rank failed");
    const uint64_t g = generation;
    if (++arrived == n) {
      arrived = 0;
      ++generation;
      cv.notify_all();
      return;
    }
    if (!cv.wait_for(lk, std::chrono::seconds(120), [&] { return generation != g || aborted; }))
      fail(QF_E_PROTOCOL, "barrier timed out");
    if (aborted) fail(QF_E_PROTOCOL, "another rank failed");
  }
  void abort() {
    std::lock_guard<std::mutex> lk(mu);
    aborted = true;
    cv.notify_all();
  }
};
struct ThreadComm : Comm {
  ThreadGroup& g;
  int r;
  ThreadComm(ThreadGroup& group, int rank) : g(group), r(rank) {}
  int rank() const override { return r; }
  int size() const override { return g.n; }
  void all_gather(const void* in, size_t n, void* out) override {
    g.slots[size_t(r)].assign(static_cast<const uint8_t*>(in), static_cast<const uint8_t*>(in) + n);
    g.barrier();
    for (int k = 0; k < g.n; ++k) {
      if (g.slots[size_t(k)].size() != n) fail(QF_E_PROTOCOL, "all_gather sizes differ");
      if (n) std::memcpy(static_cast<uint8_t*>(out) + size_t(k) * n, g.slots[size_t(k)].data(), n);
    }
    g.barrier();
  }
};

// Every rank of a block-sharded proof as a thread, each with its CPU shard;
// outputs rank 0's roots, claims and proof and whether every rank wrote the
// same three.  `claims` may be null (each rank's part of the benchmark
// claims, summed).
template <class G, class T>
int prove_sharded_threads_impl(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log,
                               uint32_t rf_bits, const T* bva, uint64_t n_values, const uint8_t* claims_in,
                               size_t claims_len, int world, uint8_t** roots, size_t* roots_len, uint8_t** claims_out,
                               size_t* claims_out_len, uint8_t** proof, size_t* proof_len, int* all_equal) {
  return guarded([&] {
    if (world < 1 || world > 256) fail(-9, "world");
    Config c;
    c.chunk_log = chunk_log;
    c.packed_log = packed_log;
    c.query_rf_bits = rf_bits;
    auto P = make_parameters<G>(shapes_of(shapes, n_shapes), c);
    validate_values(P->layout, bva, n_values);
    const BlockShards shards(P->blocks(), world);
    ThreadGroup group(world);
    const size_t n_ranks = static_cast<size_t>(world);
    std::vector<std::array<std::vector<uint8_t>, 3>> out(n_ranks);
    std::vector<std::string> errors(n_ranks);
    std::vector<std::thread> ranks;
    for (int r = 0; r < world; ++r)
      ranks.emplace_back([&, r] {
        try {
          // One rank alone takes the copy-only communicator.
          std::unique_ptr<Comm> owned;
          if (world == 1) owned = std::make_unique<LocalComm>();
          else owned = std::make_unique<ThreadComm>(group, r);
          Comm& comm = *owned;
          qf_oracle::CpuShard<G, T> shard(*P, bva, n_values, shards, r);
          ShardedBackend<G> be(*P, shard, comm);
          // Odd world sizes commit block by block (one root exchange per
          // block), even ones through commit_all (one exchange).
          std::vector<Digest> rs;
          if (world % 2) {
            for (size_t b = 0; b < P->blocks(); ++b) rs.push_back(be.commit_block(b));
          } else {
            rs = be.commit_all();
          }
          std::vector<Claim<G>> cl;
          if (claims_in) {
            ByteReader rd(claims_in, claims_len);
            for (const Shape& sh : P->layout.shapes) {
              Claim<G> x;
              for (int i = 0; i < ilog2(next_pow2(sh.rows)); ++i) x.row.push_back(rd.field<G>());
              for (int i = 0; i < ilog2(next_pow2(sh.cols)); ++i) x.col.push_back(rd.field<G>());
              x.value = rd.field<G>();
              cl.push_back(x);
            }
          } else {
            cl = sum_claims(comm, qf_oracle::evaluate_claims(*P, shard.masked.data(), n_values,
                                                             benchmark_points<G>(make_statement(*P, rs))));
          }
          const std::vector<uint8_t> wire = prove_sharded(*P, be, rs, cl);
          ByteWriter rw, cw;
          for (const auto& d : rs) rw.digest(d);
          for (const auto& x : cl) {
            for (const G& v : x.row) cw.field(v);
            for (const G& v : x.col) cw.field(v);
            cw.field(x.value);
          }
          out[size_t(r)] = {std::move(rw.out), std::move(cw.out), wire};
        } catch (const std::exception& e) {
          errors[size_t(r)] = e.what();
          group.abort();
        }
      });
    for (auto& t : ranks) t.join();
    for (int r = 0; r < world; ++r)
      if (!errors[size_t(r)].empty()) fail(QF_E_PROTOCOL, "rank " + std::to_string(r) + ": " + errors[size_t(r)]);
    *all_equal = 1;
    for (int r = 1; r < world; ++r)
      if (out[size_t(r)] != out[0]) *all_equal = 0;
    *roots = dup(out[0][0]);
    *roots_len = out[0][0].size();
    *claims_out = dup(out[0][1]);
    *claims_out_len = out[0][1].size();
    *proof = dup(out[0][2]);
    *proof_len = out[0][2].size();
  });
}
}  // namespace

extern "C" {

const char* qfo_last_error() { return g_err.c_str(); }
void qfo_free(void* p) { std::free(p); }

// Full prover over a BVA.  `claims` may be null: the benchmark points of
// main.rs:190-204 are then used.  Outputs (malloc'd): roots (blocks*32),
// claims (claims wire), proof (bincode).  `times_ms` = {commit, open}.
// F65521^8 with signed 8-bit weights; the _kb variants take KoalaBear^4 and
// signed 16-bit payloads (qafold/koalabear).
int qfo_prove(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
              const int8_t* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, uint8_t** roots,
              size_t* roots_len, uint8_t** claims_out, size_t* claims_out_len, uint8_t** proof, size_t* proof_len,
              double* times_ms) {
  return prove_impl<Fp8, int8_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in, claims_len, roots,
                                 roots_len, claims_out, claims_out_len, proof, proof_len, times_ms);
}
int qfo_prove_kb(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                 const int16_t* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, uint8_t** roots,
                 size_t* roots_len, uint8_t** claims_out, size_t* claims_out_len, uint8_t** proof, size_t* proof_len,
                 double* times_ms) {
  return prove_impl<Kb4, int16_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in, claims_len, roots,
                                  roots_len, claims_out, claims_out_len, proof, proof_len, times_ms);
}

// Commitment roots only (protocol.rs:131-185).
int qfo_commit_roots(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                     const int8_t* bva, uint64_t n_values, uint8_t* roots_out, size_t cap) {
  return commit_roots_impl<Fp8, int8_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, roots_out, cap);
}
int qfo_commit_roots_kb(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                        const int16_t* bva, uint64_t n_values, uint8_t* roots_out, size_t cap) {
  return commit_roots_impl<Kb4, int16_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, roots_out, cap);
}

// Golden vector 1: the F65521 demo bundle's proof digest and length.
int qfo_demo(uint8_t digest_out[32], uint64_t* proof_len, uint64_t* statement_json_len) {
  return demo_impl<Fp8, int8_t, uint8_t>(digest_out, proof_len, statement_json_len);
}
// Golden vector G2: the KoalaBear demo bundle (entries truncated to u16, read as i16).
int qfo_demo_kb(uint8_t digest_out[32], uint64_t* proof_len, uint64_t* statement_json_len) {
  return demo_impl<Kb4, int16_t, uint16_t>(digest_out, proof_len, statement_json_len);
}

// Golden vector 2: BLAKE2s(root || opening || decide) of the native-opening
// wire fixture (ShortQaFoldPC::new(1 << 16, 16, 2, 80), seed 0x706172616c6c656c).
int qfo_wire_fixture(uint8_t digest_out[32]) {
  return guarded([&] {
    StdRng rng = StdRng::seed_from_u64(0x706172616c6c656cull);
    auto pp = pcs_setup<F>(1u << 16, 16, 80, rng);
    std::vector<F> witness(1u << 16);
    for (auto& w : witness) w = sample_uniform(rng);
    std::vector<F> point(16);
    for (auto& p : point) p = sample_uniform(rng);
    Codeword<F> cw = encode_and_commit(pp->seq.top(), witness, pp->extension_columns, kLeafBaseDomain);
    const size_t col_log = ilog2(pp->extension_columns);
    std::vector<F> rw = tensor_weights(std::vector<F>(point.begin() + col_log, point.end()));
    std::vector<F> op = cw.project_rows(pp->top_rows(), rw);
    F claimed = inner_product(op, tensor_weights(std::vector<F>(point.begin(), point.begin() + col_log)));
    auto res = open_with_reduction(*pp, cw, point, op, claimed, rw);
    auto dec = prove_decide(*pp, res.reduction);
    auto red = verify_opening_reduction(*pp, cw.root(), point, claimed, opening_from_bytes<F>(opening_to_bytes(res.proof).data(), opening_to_bytes(res.proof).size()));
    if (!red.ok || !(red.pending == res.reduction.pending) || !verify_decide(*pp, red, dec)) fail(-3, "fixture self-verification");
    Blake2s h;
    h.update(cw.root());
    h.update(opening_to_bytes(res.proof));
    h.update(decide_to_bytes(dec));
    Digest d = h.finalize();
    std::memcpy(digest_out, d.data(), 32);
  });
}

// Independent verification of a proof (protocol.rs:266-320).
int qfo_verify(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
               const uint8_t* roots, const uint8_t* claims_in, size_t claims_len, const uint8_t* proof, size_t proof_len) {
  return verify_impl<Fp8>(shapes, n_shapes, chunk_log, packed_log, rf_bits, roots, claims_in, claims_len, proof, proof_len);
}
int qfo_verify_kb(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                  const uint8_t* roots, const uint8_t* claims_in, size_t claims_len, const uint8_t* proof, size_t proof_len) {
  return verify_impl<Kb4>(shapes, n_shapes, chunk_log, packed_log, rf_bits, roots, claims_in, claims_len, proof, proof_len);
}

// LogUp range audit of `n` BVA values (multiplicities: 256 or 65536 bins).
int qfo_range_audit(const int8_t* values, uint64_t n, const uint8_t seed[32], uint64_t* mult, uint8_t alpha[16],
                    uint8_t lhs[16], uint8_t rhs[16]) {
  return range_audit_impl<Fp8, int8_t>(values, n, seed, mult, alpha, lhs, rhs);
}
int qfo_range_audit_kb(const int16_t* values, uint64_t n, const uint8_t seed[32], uint64_t* mult, uint8_t alpha[16],
                       uint8_t lhs[16], uint8_t rhs[16]) {
  return range_audit_impl<Kb4, int16_t>(values, n, seed, mult, alpha, lhs, rhs);
}

// One rank of a block-sharded proof; `gather(ctx, in, n, out)` is the
// all-gather over the `world` ranks (out = every rank's n bytes, in rank
// order) and `reduce(ctx, data, n)`, which may be null, the sum of n 64-bit
// integers over the ranks; both return 0 on success.  Outputs as qfo_prove's.
int qfo_prove_sharded(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                      const int8_t* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, int rank, int world,
                      CallbackComm::Fn gather, CallbackComm::ReduceFn reduce, void* comm_ctx, uint8_t** roots,
                      size_t* roots_len, uint8_t** claims_out, size_t* claims_out_len, uint8_t** proof,
                      size_t* proof_len) {
  return prove_sharded_impl<Fp8, int8_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in,
                                         claims_len, rank, world, gather, reduce, comm_ctx, roots, roots_len, claims_out,
                                         claims_out_len, proof, proof_len);
}
int qfo_prove_sharded_kb(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                         const int16_t* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, int rank,
                         int world, CallbackComm::Fn gather, CallbackComm::ReduceFn reduce, void* comm_ctx,
                         uint8_t** roots, size_t* roots_len, uint8_t** claims_out, size_t* claims_out_len,
                         uint8_t** proof, size_t* proof_len) {
  return prove_sharded_impl<Kb4, int16_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in,
                                          claims_len, rank, world, gather, reduce, comm_ctx, roots, roots_len, claims_out,
                                          claims_out_len, proof, proof_len);
}

// The compiled query in dense form beside its claim, evaluation and cross
// terms (layout above tbv_dense_impl), for a check against the definitions.
int qfo_tbv_dense(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                  const int8_t* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, uint32_t stride,
                  uint8_t** out, size_t* out_len) {
  return tbv_dense_impl<Fp8, int8_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in,
                                     claims_len, stride, out, out_len);
}
int qfo_tbv_dense_kb(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                     const int16_t* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, uint32_t stride,
                     uint8_t** out, size_t* out_len) {
  return tbv_dense_impl<Kb4, int16_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in,
                                      claims_len, stride, out, out_len);
}

// The extension fields' product, inverse and Frobenius step, element-wise.
int qfo_field_ops(const uint8_t* a, const uint8_t* b, size_t n, uint8_t* prod, uint8_t* inv, uint8_t* frob) {
  return field_ops_impl<Fp8>(a, b, n, prod, inv, frob);
}
int qfo_field_ops_kb(const uint8_t* a, const uint8_t* b, size_t n, uint8_t* prod, uint8_t* inv, uint8_t* frob) {
  return field_ops_impl<Kb4>(a, b, n, prod, inv, frob);
}

// Single-block packed PCS open and verify over canonical base values.
int qfo_packed_open(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], const int32_t* values,
                    const uint8_t* point, const uint8_t* ctx, size_t ctx_len, uint8_t root[32], uint8_t value[16],
                    uint8_t** proof, size_t* proof_len) {
  return packed_open_impl<Fp8>(log_n, columns, bits, seed, values, point, ctx, ctx_len, root, value, proof, proof_len);
}
int qfo_packed_open_kb(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], const int32_t* values,
                       const uint8_t* point, const uint8_t* ctx, size_t ctx_len, uint8_t root[32], uint8_t value[16],
                       uint8_t** proof, size_t* proof_len) {
  return packed_open_impl<Kb4>(log_n, columns, bits, seed, values, point, ctx, ctx_len, root, value, proof, proof_len);
}
int qfo_packed_verify(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], const uint8_t root[32],
                      const uint8_t* point, const uint8_t value[16], const uint8_t* proof, size_t proof_len,
                      const uint8_t* ctx, size_t ctx_len) {
  return packed_verify_impl<Fp8>(log_n, columns, bits, seed, root, point, value, proof, proof_len, ctx, ctx_len);
}
int qfo_packed_verify_kb(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], const uint8_t root[32],
                         const uint8_t* point, const uint8_t value[16], const uint8_t* proof, size_t proof_len,
                         const uint8_t* ctx, size_t ctx_len) {
  return packed_verify_impl<Kb4>(log_n, columns, bits, seed, root, point, value, proof, proof_len, ctx, ctx_len);
}

// Batched packed PCS open and verify over canonical base values.
int qfo_packed_open_batch(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], uint32_t blocks,
                          const int32_t* values, const uint8_t* point, const uint8_t* ctx, size_t ctx_len, uint8_t* roots,
                          uint8_t value[16], uint8_t** proof, size_t* proof_len) {
  return packed_open_batch_impl<Fp8>(log_n, columns, bits, seed, blocks, values, point, ctx, ctx_len, roots, value, proof,
                                     proof_len);
}
int qfo_packed_open_batch_kb(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], uint32_t blocks,
                             const int32_t* values, const uint8_t* point, const uint8_t* ctx, size_t ctx_len,
                             uint8_t* roots, uint8_t value[16], uint8_t** proof, size_t* proof_len) {
  return packed_open_batch_impl<Kb4>(log_n, columns, bits, seed, blocks, values, point, ctx, ctx_len, roots, value, proof,
                                     proof_len);
}
int qfo_packed_verify_batch(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], uint32_t blocks,
                            const uint8_t* roots, const uint8_t* point, uint32_t point_len, const uint8_t value[16],
                            const uint8_t* proof, size_t proof_len, const uint8_t* ctx, size_t ctx_len) {
  return packed_verify_batch_impl<Fp8>(log_n, columns, bits, seed, blocks, roots, point, point_len, value, proof, proof_len,
                                       ctx, ctx_len);
}
int qfo_packed_verify_batch_kb(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t seed[32], uint32_t blocks,
                               const uint8_t* roots, const uint8_t* point, uint32_t point_len, const uint8_t value[16],
                               const uint8_t* proof, size_t proof_len, const uint8_t* ctx, size_t ctx_len) {
  return packed_verify_batch_impl<Kb4>(log_n, columns, bits, seed, blocks, roots, point, point_len, value, proof, proof_len,
                                       ctx, ctx_len);
}

// Codeword-fold binding made under one set of block weights, checked under another.
int qfo_codeword_fold(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t pcs_seed[32], uint32_t blocks,
                      const int32_t* values, const uint32_t* fold_w, const uint8_t seed[32], const uint32_t* check_w,
                      int* accepted) {
  return codeword_fold_impl<Fp8>(log_n, columns, bits, pcs_seed, blocks, values, fold_w, seed, check_w, accepted);
}
int qfo_codeword_fold_kb(uint32_t log_n, uint32_t columns, uint32_t bits, const uint8_t pcs_seed[32], uint32_t blocks,
                         const int32_t* values, const uint32_t* fold_w, const uint8_t seed[32], const uint32_t* check_w,
                         int* accepted) {
  return codeword_fold_impl<Kb4>(log_n, columns, bits, pcs_seed, blocks, values, fold_w, seed, check_w, accepted);
}

// The prover without the weights' layout check (outputs: the proof bytes).
int qfo_prove_unchecked(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log, uint32_t rf_bits,
                        const int8_t* bva, uint64_t n_values, const uint8_t* claims_in, size_t claims_len, uint8_t** proof,
                        size_t* proof_len) {
  return prove_unchecked_impl<Fp8, int8_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in,
                                           claims_len, proof, proof_len);
}
int qfo_prove_unchecked_kb(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log,
                           uint32_t rf_bits, const int16_t* bva, uint64_t n_values, const uint8_t* claims_in,
                           size_t claims_len, uint8_t** proof, size_t* proof_len) {
  return prove_unchecked_impl<Kb4, int16_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values, claims_in,
                                            claims_len, proof, proof_len);
}

// BLAKE2s-256 of `n` bytes fed to one hasher in pieces that end at the
// `n_cuts` ascending offsets `cuts` (then the rest).
int qfo_blake2s_stream(const uint8_t* data, size_t n, const uint64_t* cuts, size_t n_cuts, uint8_t out[32]) {
  return guarded([&] {
    Blake2s h;
    size_t at = 0;
    for (size_t i = 0; i < n_cuts; ++i) {
      if (cuts[i] < at || cuts[i] > n) fail(-9, "cuts");
      h.update(data + at, size_t(cuts[i] - at));
      at = size_t(cuts[i]);
    }
    h.update(data + at, n - at);
    const Digest d = h.finalize();
    std::memcpy(out, d.data(), 32);
  });
}
// One compression of `block` into the state h (t = the byte count after the
// block, `last` the final-block flag) by the scalar or the SSSE3 path.
int qfo_blake2s_compress(const uint32_t h_in[8], const uint8_t block[64], uint64_t t, int last, int ssse3,
                         uint32_t h_out[8]) {
  return guarded([&] {
    uint32_t h[8];
    std::memcpy(h, h_in, sizeof h);
#if defined(__x86_64__)
    if (ssse3) {
      if (!__builtin_cpu_supports("ssse3")) fail(-9, "no SSSE3 on this host");
      blake2s_compress_ssse3(h, block, t, last != 0);
    } else {
      blake2s_compress_scalar(h, block, t, last != 0);
    }
#else
    if (ssse3) fail(-9, "no SSSE3 on this host");
    blake2s_compress_scalar(h, block, t, last != 0);
#endif
    std::memcpy(h_out, h, sizeof h);
  });
}

// The setup's generator (rand 0.8 StdRng) driven by a list of draws: a
// positive op k is fill_bytes of k bytes, -1 is next_u32 and -2 next_u64
// (little-endian); the outputs are concatenated into `out`.  With
// `use_u64` the generator is StdRng::seed_from_u64(seed_u64), else
// StdRng::from_seed(seed).
int qfo_stdrng(const uint8_t seed[32], uint64_t seed_u64, int use_u64, const int32_t* ops, size_t n_ops, uint8_t* out,
               size_t cap) {
  return guarded([&] {
    std::array<uint8_t, 32> sd{};
    if (seed) std::memcpy(sd.data(), seed, 32);
    StdRng rng = use_u64 ? StdRng::seed_from_u64(seed_u64) : StdRng(sd);
    size_t at = 0;
    auto room = [&](size_t k) { if (at + k > cap) fail(-9, "output buffer too small"); };
    for (size_t i = 0; i < n_ops; ++i) {
      if (ops[i] > 0) {
        room(size_t(ops[i]));
        rng.fill_bytes(out + at, size_t(ops[i]));
        at += size_t(ops[i]);
      } else if (ops[i] == -1) {
        room(4);
        const uint32_t v = rng.next_u32();
        for (int j = 0; j < 4; ++j) out[at++] = uint8_t(v >> (8 * j));
      } else if (ops[i] == -2) {
        room(8);
        const uint64_t v = rng.next_u64();
        for (int j = 0; j < 8; ++j) out[at++] = uint8_t(v >> (8 * j));
      } else {
        fail(-9, "unknown draw");
      }
    }
  });
}

// The query counts of every level of a packed PCS's code sequence.
int qfo_query_counts(uint32_t log_n, uint32_t columns, uint32_t bits, uint64_t* rows, size_t cap, size_t* levels,
                     double* card_log2) {
  return query_counts_impl<Fp8>(log_n, columns, bits, rows, cap, levels, card_log2);
}
int qfo_query_counts_kb(uint32_t log_n, uint32_t columns, uint32_t bits, uint64_t* rows, size_t cap, size_t* levels,
                        double* card_log2) {
  return query_counts_impl<Kb4>(log_n, columns, bits, rows, cap, levels, card_log2);
}

// The host layout of `shapes` (Layout::new, layout.rs:34-155): per bucket,
// in layout order, matrix, offset, row offset, column offset, rows, columns,
// physical rows, physical columns; then active and logical.
int qfo_layout(const uint64_t* shapes, size_t n_shapes, uint64_t* out, size_t cap, size_t* n_buckets) {
  return guarded([&] {
    const Layout L = make_layout(shapes_of(shapes, n_shapes));
    if (cap < 8 * L.buckets.size() + 2) fail(-9, "output buffer too small");
    size_t at = 0;
    for (const Bucket& b : L.buckets)
      for (size_t v : {b.matrix, b.offset, b.row_offset, b.col_offset, b.rows, b.cols, b.physical_rows, b.physical_cols})
        out[at++] = v;
    out[at++] = L.active;
    out[at++] = L.logical;
    *n_buckets = L.buckets.size();
  });
}

// Every rank of a block-sharded proof as a thread of this process.
int qfo_prove_sharded_threads(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log,
                              uint32_t rf_bits, const int8_t* bva, uint64_t n_values, const uint8_t* claims_in,
                              size_t claims_len, int world, uint8_t** roots, size_t* roots_len, uint8_t** claims_out,
                              size_t* claims_out_len, uint8_t** proof, size_t* proof_len, int* all_equal) {
  return prove_sharded_threads_impl<Fp8, int8_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values,
                                                 claims_in, claims_len, world, roots, roots_len, claims_out,
                                                 claims_out_len, proof, proof_len, all_equal);
}
int qfo_prove_sharded_threads_kb(const uint64_t* shapes, size_t n_shapes, uint32_t chunk_log, uint32_t packed_log,
                                 uint32_t rf_bits, const int16_t* bva, uint64_t n_values, const uint8_t* claims_in,
                                 size_t claims_len, int world, uint8_t** roots, size_t* roots_len, uint8_t** claims_out,
                                 size_t* claims_out_len, uint8_t** proof, size_t* proof_len, int* all_equal) {
  return prove_sharded_threads_impl<Kb4, int16_t>(shapes, n_shapes, chunk_log, packed_log, rf_bits, bva, n_values,
                                                  claims_in, claims_len, world, roots, roots_len, claims_out,
                                                  claims_out_len, proof, proof_len, all_equal);
}

// The top QA code of a packed PCS over 2^log_n base values (columns 32,
// `bits` of security, setup seed 0x51..): its message length R, its alpha
// table alphas[1] (R elements) and the codeword of the R-element message
// column `message` (2R elements), for a check against the encoding's
// definition (qafold_short.rs:975-1002).
int qfo_encode_column(int kb, uint32_t log_n, uint32_t bits, const uint8_t* message, size_t message_len, uint8_t* alpha,
                      uint8_t* codeword, size_t* rows) {
  return guarded([&] {
    auto run = [&](auto tag) {
      using G = decltype(tag);
      std::array<uint8_t, 32> sd;
      sd.fill(0x51);
      PackedPcs<G> pcs = PackedPcs<G>::create(log_n, 32, bits, sd);
      const QaCode<G>& code = pcs.pp->seq.top();
      *rows = code.message_len;
      if (message_len != code.message_len) fail(-9, "message length");
      std::vector<G> msg(message_len), out(code.codeword_len());
      ByteReader r(message, 16 * message_len);
      for (auto& m : msg) m = r.field<G>();
      code.encode_into(msg.data(), out.data());
      for (size_t i = 0; i < message_len; ++i) code.alphas[1][i].to_bytes(alpha + 16 * i);
      for (size_t i = 0; i < out.size(); ++i) out[i].to_bytes(codeword + 16 * i);
    };
    if (kb) run(Kb4{});
    else run(Fp8{});
  });
}

}  // extern "C"
