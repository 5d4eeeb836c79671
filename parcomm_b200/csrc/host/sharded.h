// Block-sharded proof: one proof over a BVA whose PCS blocks are spread over
// several ranks (one process per device).
//
// The blocks are independent until the batch opening folds them: each is
// committed on its own (protocol.rs:168-178), projected on its own
// (packed_batch.rs:161-163) and enters the fold through one weight
// (packed_batch.rs:213-236).  Rank r holds the contiguous run of blocks
// [B r / N, B (r + 1) / N).  Every value the prover derives from the weights
// is linear in them, so each rank computes the part that its own blocks
// contribute and the parts are summed over the ranks before the transcript
// absorbs them:
//   - commit: each rank commits the blocks it holds; the roots are gathered;
//   - EO (eo.rs:97-181): the cross terms, the witness-query dot product,
//     both cross elements of every binary round and the terminal witness
//     value.  Each rank keeps and folds its own part of the witness; the
//     query depends on the claims alone and is whole on every rank;
//   - batch opening: the blocks' lane sums and the folded values (m field
//     elements, the one large exchange).  The folded commit, the sumcheck,
//     the native opening and Decide then run on every rank over the same
//     data;
//   - binding (qafold_short_batch.rs:77-160): each rank writes the sampled
//     rows of its own blocks and the pieces are joined in block order.
// Every challenge is thus derived from values that all ranks hold byte for
// byte, and the unchanged drivers (eo_prove, open_batch) write on every rank
// the proof that a single rank holding all blocks writes.
#pragma once
#include <cstring>
#include <memory>
#include <vector>

#include "protocol.h"

namespace qf {

// The collectives the sharded proof uses.
struct Comm {
  virtual ~Comm() {}
  virtual int rank() const = 0;
  virtual int size() const = 0;
  // out[r n, (r + 1) n) <- rank r's n bytes `in`; every rank passes the same n.
  virtual void all_gather(const void* in, size_t n, void* out) = 0;
  // data[i] <- the sum over the ranks of data[i] (every rank passes the same
  // n; the sums used here stay below 2^63).  The form of an integer
  // all-reduce (NCCL's uint64 sum); by default built on all_gather.
  virtual void all_reduce_sum(uint64_t* data, size_t n) {
    std::vector<uint64_t> all(n * size_t(size()));
    all_gather(data, 8 * n, all.data());
    for (size_t i = 0; i < n; ++i) {
      uint64_t t = 0;
      for (int k = 0; k < size(); ++k) t += all[size_t(k) * n + i];
      data[i] = t;
    }
  }
};

// A Comm over C callbacks, the form a caller outside C++ provides (MPI,
// torch.distributed, NCCL over host buffers).  Each callback returns 0 on
// success; without `reduce`, sums go through the gather.
struct CallbackComm : Comm {
  using Fn = int (*)(void* ctx, const void* in, size_t n, void* out);
  using ReduceFn = int (*)(void* ctx, uint64_t* data, size_t n);
  int r, n;
  Fn fn;
  ReduceFn reduce;
  void* ctx;
  CallbackComm(int rank, int size, Fn f, void* c, ReduceFn red = nullptr) : r(rank), n(size), fn(f), reduce(red), ctx(c) {
    if (size < 1 || rank < 0 || rank >= size || !f) fail(QF_E_ARGUMENT, "communicator rank/size/callback");
  }
  int rank() const override { return r; }
  int size() const override { return n; }
  void all_gather(const void* in, size_t bytes, void* out) override {
    if (fn(ctx, in, bytes, out) != 0) fail(QF_E_PROTOCOL, "all_gather callback failed");
  }
  void all_reduce_sum(uint64_t* data, size_t count) override {
    if (!reduce) return Comm::all_reduce_sum(data, count);
    if (reduce(ctx, data, count) != 0) fail(QF_E_PROTOCOL, "all_reduce callback failed");
  }
};

// One rank alone: the gather is a copy.
struct LocalComm : Comm {
  int rank() const override { return 0; }
  int size() const override { return 1; }
  void all_gather(const void* in, size_t n, void* out) override { if (n) std::memcpy(out, in, n); }
};

// Rank r holds blocks [first(r), first(r + 1)).
struct BlockShards {
  size_t blocks = 0;
  int ranks = 1;
  BlockShards(size_t b, int n) : blocks(b), ranks(n) {
    if (n < 1 || size_t(n) > b) fail(QF_E_ARGUMENT, "block shards: need 1 <= ranks <= blocks");
  }
  size_t first(int r) const { return blocks * size_t(r) / size_t(ranks); }
  bool holds(int r, size_t b) const { return b >= first(r) && b < first(r + 1); }
  int owner(size_t b) const {
    int r = 0;
    while (!holds(r, b)) ++r;
    return r;
  }
};

// Sum over the ranks of each rank's vector `part` (the same length on every
// rank): the canonical coefficients (each below p < 2^31) are summed as
// 64-bit integers, which cannot overflow below 2^32 ranks, and reduced mod p
// once, so every rank gets the same canonical elements.
template <class F>
std::vector<F> sum_over_ranks(Comm& c, const std::vector<F>& part) {
  if (part.empty() || c.size() == 1) return part;
  constexpr int kD = int(sizeof(F::c) / sizeof(typename F::Coeff));  // coefficients per element
  std::vector<uint64_t> wide(part.size() * kD);
  for (size_t i = 0; i < part.size(); ++i)
    for (int k = 0; k < kD; ++k) wide[i * kD + k] = uint64_t(part[i].c[k]);
  c.all_reduce_sum(wide.data(), wide.size());
  std::vector<F> total(part.size());
  const uint64_t p = F::modulus_u64();
  for (size_t i = 0; i < part.size(); ++i)
    for (int k = 0; k < kD; ++k) total[i].c[k] = typename F::Coeff(wide[i * kD + k] % p);
  return total;
}

// Every rank's byte string, of any length, in rank order.
inline std::vector<std::vector<uint8_t>> gather_bytes(Comm& c, const std::vector<uint8_t>& mine) {
  const size_t n = size_t(c.size());
  const auto len = le64(mine.size());
  std::vector<uint8_t> lens(8 * n);
  c.all_gather(len.data(), 8, lens.data());
  std::vector<uint64_t> each(n);
  uint64_t widest = 0;
  for (size_t k = 0; k < n; ++k) {
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v |= uint64_t(lens[8 * k + i]) << (8 * i);
    each[k] = v;
    widest = std::max(widest, v);
  }
  std::vector<std::vector<uint8_t>> out(n);
  if (widest == 0) return out;
  std::vector<uint8_t> padded(mine);
  padded.resize(widest, 0);
  std::vector<uint8_t> all(widest * n);
  c.all_gather(padded.data(), widest, all.data());
  for (size_t k = 0; k < n; ++k) out[k].assign(all.begin() + k * widest, all.begin() + k * widest + each[k]);
  return out;
}

// What one rank computes over the blocks it holds.  Each value that is a
// sum over the weights (the lane sums, the EO cross terms, dot product,
// round cross elements and terminal witness value, the folded values) is
// this rank's part of it: blocks it does not hold count as zero.  The
// equality weights, the query and everything after the fold exchange are
// whole on every rank.
template <class F>
struct ShardBackend : EoBackend<F> {
  // Commit held block b; keeps its codeword for the binding rows.
  virtual Digest commit_block(size_t b) = 0;
  // Weights <- eq(outer); lane sums of every block (zero for blocks not held).
  virtual std::vector<std::vector<F>> project_blocks(const std::vector<F>& outer, size_t blocks) = 0;
  virtual void apply_images(const std::vector<F>& images) = 0;
  // This rank's part of sum_b fold[b] * packed(b, .).
  virtual std::vector<F> fold_part(const std::vector<F>& fold_weights) = 0;
  // The summed folded values: keep them for the sumcheck, commit them, return the root.
  virtual Digest commit_folded(std::vector<F> values) = 0;
  virtual void sumcheck_message(F m[2]) = 0;
  virtual void sumcheck_fold(F ch) = 0;
  virtual F sumcheck_final_value() = 0;
  virtual F sumcheck_final_weight() = 0;
  // Sampled rows of held block b (whose root must be `root`), and of the folded codeword.
  virtual void write_block_rows(ByteWriter& w, size_t b, const RowSelection& sel, const Digest& root) = 0;
  virtual void write_folded_rows(ByteWriter& w, const RowSelection& sel) = 0;
  virtual const CodewordView<F>& folded_codeword() = 0;
  virtual std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& row_weights) = 0;
  virtual TopRoundAccel<F>* top_round_accel() { return nullptr; }
  virtual DecideAccel<F>* decide_accel() { return nullptr; }
};

// The batch-opening and EO backends that the protocol drivers see: one
// rank's shard plus the sums over the ranks.
template <class F>
class ShardedBackend : public Backend<F>, public EoBackend<F> {
 public:
  ShardedBackend(const Parameters<F>& P, ShardBackend<F>& shard, Comm& comm)
      : P_(P), s_(shard), c_(comm), shards_(P.blocks(), comm.size()) {}

  const BlockShards& shards() const { return shards_; }
  bool holds(size_t b) const { return shards_.holds(c_.rank(), b); }

  // Commits the held blocks, then gathers every block's root.
  std::vector<Digest> commit_all() {
    std::vector<uint8_t> mine(32 * P_.blocks(), 0);
    for (size_t b = shards_.first(c_.rank()); b < shards_.first(c_.rank() + 1); ++b) {
      const Digest d = s_.commit_block(b);
      std::memcpy(mine.data() + 32 * b, d.data(), 32);
    }
    std::vector<uint8_t> all(mine.size() * size_t(c_.size()));
    c_.all_gather(mine.data(), mine.size(), all.data());
    std::vector<Digest> roots(P_.blocks());
    for (size_t b = 0; b < roots.size(); ++b)
      std::memcpy(roots[b].data(), all.data() + size_t(shards_.owner(b)) * mine.size() + 32 * b, 32);
    return roots;
  }

  // ---- Backend
  Digest commit_block(size_t b) override {
    Digest d{};
    if (holds(b)) d = s_.commit_block(b);
    std::vector<uint8_t> all(32 * size_t(c_.size()));
    c_.all_gather(d.data(), 32, all.data());
    std::memcpy(d.data(), all.data() + 32 * size_t(shards_.owner(b)), 32);
    return d;
  }
  std::vector<std::vector<F>> project_blocks(const std::vector<F>& outer, size_t blocks) override {
    std::vector<std::vector<F>> parts = s_.project_blocks(outer, blocks);
    check(parts.size() == blocks, "shard lane sums: block count");
    std::vector<F> flat;
    for (const auto& p : parts) {
      check(p.size() == size_t(F::kLanes), "shard lane sums: lane count");
      flat.insert(flat.end(), p.begin(), p.end());
    }
    flat = sum_over_ranks(c_, flat);
    for (size_t b = 0; b < blocks; ++b) parts[b].assign(flat.begin() + b * F::kLanes, flat.begin() + (b + 1) * F::kLanes);
    return parts;
  }
  void apply_images(const std::vector<F>& images) override { s_.apply_images(images); }
  Digest fold_and_commit(const std::vector<F>& fold_weights) override {
    return s_.commit_folded(sum_over_ranks(c_, s_.fold_part(fold_weights)));
  }
  void sumcheck_message(F m[2]) override { s_.sumcheck_message(m); }
  void sumcheck_fold(F ch) override { s_.sumcheck_fold(ch); }
  F sumcheck_final_value() override { return s_.sumcheck_final_value(); }
  F sumcheck_final_weight() override { return s_.sumcheck_final_weight(); }
  // The "QAFOLDB1" payload: block count, each block's rows in block order,
  // then the folded codeword's rows.
  std::vector<uint8_t> binding_rows(const RowSelection& sel, const std::vector<Digest>& roots) override {
    check(roots.size() == P_.blocks(), "binding: root count");
    ByteWriter mine;
    for (size_t b = shards_.first(c_.rank()); b < shards_.first(c_.rank() + 1); ++b)
      s_.write_block_rows(mine, b, sel, roots[b]);
    std::vector<std::vector<uint8_t>> pieces = gather_bytes(c_, mine.out);
    ByteWriter w;
    w.bytes("QAFOLDB1", 8);
    w.len(roots.size());
    for (const auto& p : pieces) w.bytes(p.data(), p.size());
    s_.write_folded_rows(w, sel);
    return std::move(w.out);
  }
  const CodewordView<F>& folded_codeword() override { return s_.folded_codeword(); }
  std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& row_weights) override {
    return s_.folded_opening(point, col_log, row_weights);
  }
  TopRoundAccel<F>* top_round_accel() override { return s_.top_round_accel(); }
  DecideAccel<F>* decide_accel() override { return s_.decide_accel(); }

  // ---- EoBackend
  void cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) override {
    s_.cross_terms(q, stride, pos, neg);
    check(pos.size() == neg.size(), "shard cross terms");
    std::vector<F> both(pos);
    both.insert(both.end(), neg.begin(), neg.end());
    both = sum_over_ranks(c_, both);
    pos.assign(both.begin(), both.begin() + pos.size());
    neg.assign(both.begin() + pos.size(), both.end());
  }
  F eo_build(const Query<F>& q, F challenge, F inverse, size_t logical, size_t stride) override {
    return sum_over_ranks(c_, std::vector<F>{s_.eo_build(q, challenge, inverse, logical, stride)})[0];
  }
  std::array<F, 2> eo_round_cross() override {
    const std::array<F, 2> part = s_.eo_round_cross();
    const std::vector<F> t = sum_over_ranks(c_, std::vector<F>{part[0], part[1]});
    return {t[0], t[1]};
  }
  void eo_round_fold(F inv, F ch) override { s_.eo_round_fold(inv, ch); }
  std::array<F, 2> eo_terminal() override {
    const std::array<F, 2> part = s_.eo_terminal();
    return {sum_over_ranks(c_, std::vector<F>{part[0]})[0], part[1]};
  }

 private:
  const Parameters<F>& P_;
  ShardBackend<F>& s_;
  Comm& c_;
  BlockShards shards_;
};

// Claims from each rank's parts: a claim's value is a sum over the weights
// (tbv.rs:143-185), so the parts add up; the points are the same on every rank.
template <class F>
std::vector<Claim<F>> sum_claims(Comm& c, std::vector<Claim<F>> parts) {
  std::vector<F> v;
  for (const Claim<F>& cl : parts) v.push_back(cl.value);
  v = sum_over_ranks(c, v);
  for (size_t i = 0; i < parts.size(); ++i) parts[i].value = v[i];
  return parts;
}

// The outer prover (protocol.rs:201-263) over block shards, on every rank:
// the statement transcript and query, the EO, the batch opening, the proof
// wire.  `roots` come from commit_all and `claims` are whole.  A BVA of one
// block has nothing to shard; it is proved by one rank.
template <class F>
std::vector<uint8_t> prove_sharded(const Parameters<F>& P, ShardedBackend<F>& be, const std::vector<Digest>& roots,
                                   const std::vector<Claim<F>>& claims) {
  check(roots.size() == P.blocks() && roots.size() >= 2, "sharded proof: needs the roots of two or more blocks");
  const Commitment st = make_statement(P, roots);
  Transcript<F> t = statement_transcript(P, st, claims);
  const Query<F> q = compile(P.layout, claims, t);
  auto [eo, term] = eo_prove<F>(be, P.layout.logical, size_t(1) << P.config.packed_log, q, t);
  const std::vector<uint8_t> ctx = opening_context<F>(t.state, 0);
  BatchOpening<F> op = open_batch(P.pcs, be, roots, term.point_msb, ctx);
  check(op.claimed_value * term.scale == term.value, "QAFold/EO terminal mismatch");
  Proof<F> pr;
  pr.eo = std::move(eo);
  pr.opening_value = op.claimed_value;
  pr.opening_proof = std::move(op.wire);
  return proof_to_bytes(pr);
}

}  // namespace qf
