// The field-specific half of the extern "C" boundary (see capi.cu): the
// bodies of commit, claims, prove and verify for the field picked by
// field_select.h.  This file is compiled once per field (capi_field_kb.cu
// defines QF_FIELD_KB and includes it); each compilation exports its table as
// QFB_NS::kFieldApi.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <string>

#include "capi_internal.h"
#include "gpu_backend.cuh"
#include "host/range_audit.h"
#include "host/sharded.h"

namespace QFB_NS {
namespace {

const Parameters<F>& params_of(const qf_params* p) { return *static_cast<const Parameters<F>*>(p->P.get()); }

// Any zero-padding entry that is nonzero sets the flag (Layout::validate_values,
// layout.rs:136-155).  Segments are at most kZeroPiece bytes; a CTA checks one
// with 16-byte loads over its aligned middle and byte loads at the ends.
constexpr uint64_t kZeroPiece = 4096;
__global__ void k_check_zero_segments(const uint8_t* __restrict__ bva, const uint64_t* __restrict__ seg, uint32_t n_seg,
                                      unsigned int* __restrict__ flag) {
  bool bad = false;
  for (uint32_t s = blockIdx.x; s < n_seg; s += gridDim.x) {
    const uint64_t a = seg[2 * s], b = seg[2 * s + 1];
    const uint64_t a16 = (a + 15) & ~uint64_t(15), b16 = b & ~uint64_t(15);
    if (a16 >= b16) {
      for (uint64_t i = a + threadIdx.x; i < b; i += blockDim.x) bad |= bva[i] != 0;
    } else {
      for (uint64_t i = a + threadIdx.x; i < a16; i += blockDim.x) bad |= bva[i] != 0;
      for (uint64_t i = b16 + threadIdx.x; i < b; i += blockDim.x) bad |= bva[i] != 0;
      for (uint64_t i = a16 + 16 * uint64_t(threadIdx.x); i < b16; i += 16 * uint64_t(blockDim.x)) {
        const uint4 u = *reinterpret_cast<const uint4*>(bva + i);
        bad |= (u.x | u.y | u.z | u.w) != 0;
      }
    }
  }
  if (bad) atomicOr(flag, 1u);
}


// The entries of the layout's zero padding (Layout::validate_values,
// layout.rs:136-155) inside [lo, hi), as byte ranges relative to lo, cut into
// pieces of at most kZeroPiece bytes.
static std::vector<uint64_t> padding_segments(const Parameters<F>& P, uint64_t lo, uint64_t hi) {
  std::vector<uint64_t> runs;
  auto add_run = [&](uint64_t a, uint64_t e) {
    a = std::max(a, lo);
    e = std::min(e, hi);
    if (a >= e) return;
    if (!runs.empty() && runs.back() == a) runs.back() = e;  // merge contiguous runs
    else { runs.push_back(a); runs.push_back(e); }
  };
  for (const Bucket& b : P.layout.buckets) {
    if (b.offset + b.rows * b.cols <= lo || b.offset >= hi) continue;
    if (b.physical_cols < b.cols)  // the padded tail of every real row
      for (size_t r = 0; r < b.physical_rows; ++r) add_run(b.offset + r * b.cols + b.physical_cols, b.offset + (r + 1) * b.cols);
    add_run(b.offset + b.physical_rows * b.cols, b.offset + b.rows * b.cols);  // padding rows
  }
  std::vector<uint64_t> seg;
  for (size_t i = 0; i < runs.size(); i += 2)
    for (uint64_t a = (runs[i] - lo) * sizeof(W); a < (runs[i + 1] - lo) * sizeof(W); a += kZeroPiece) {
      seg.push_back(a);
      seg.push_back(std::min<uint64_t>(a + kZeroPiece, (runs[i + 1] - lo) * sizeof(W)));
    }
  return seg;
}

// A side stream for the weight transfer, with one event per block.
struct CopyPipeline {
  cudaStream_t stream = nullptr;
  cudaEvent_t begin = nullptr, end = nullptr;
  std::vector<cudaEvent_t> landed;
  explicit CopyPipeline(size_t blocks) : landed(blocks, nullptr) {
    QF_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    QF_CK(cudaEventCreate(&begin));
    QF_CK(cudaEventCreate(&end));
    for (auto& e : landed) QF_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  ~CopyPipeline() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& e : landed)
      if (e) cudaEventDestroy(e);
    if (begin) cudaEventDestroy(begin);
    if (end) cudaEventDestroy(end);
    if (stream) cudaStreamDestroy(stream);
  }
  CopyPipeline(const CopyPipeline&) = delete;
  CopyPipeline& operator=(const CopyPipeline&) = delete;
};

struct FieldCommitted : qf_committed_state {
  cudaStream_t stream = nullptr;
  DBuf<W> bva;                       // resident weights
  std::unique_ptr<BlockStream> src;  // or streamed weights
  uint64_t active = 0;
  std::unique_ptr<GpuBackend> be;
  std::vector<Digest> roots;
  double commit_ms = 0, upload_ms = 0;
  ~FieldCommitted() override {
    be.reset();
    src.reset();
    bva.reset();
    if (stream) cudaStreamDestroy(stream);
  }
};

static std::vector<Claim<F>> parse_claims(const Parameters<F>& P, const uint8_t* d, size_t n, bool with_value) {
  std::vector<Claim<F>> claims;
  ByteReader r(d, n);
  for (const Shape& s : P.layout.shapes) {
    Claim<F> c;
    for (int i = 0; i < ilog2(next_pow2(s.rows)); ++i) c.row.push_back(r.field<F>());
    for (int i = 0; i < ilog2(next_pow2(s.cols)); ++i) c.col.push_back(r.field<F>());
    c.value = with_value ? r.field<F>() : F::zero();
    claims.push_back(std::move(c));
  }
  if (!r.empty()) fail(QF_E_ARGUMENT, "claims length mismatch");
  return claims;
}
static std::vector<uint8_t> write_claims(const std::vector<Claim<F>>& claims, bool with_value) {
  ByteWriter w;
  for (const auto& c : claims) {
    for (const F& v : c.row) w.field(v);
    for (const F& v : c.col) w.field(v);
    if (with_value) w.field(c.value);
  }
  return std::move(w.out);
}
static std::vector<Digest> roots_from(const qf_params* p, const uint8_t* roots) {
  std::vector<Digest> out(params_of(p).blocks());
  for (size_t b = 0; b < out.size(); ++b) std::memcpy(out[b].data(), roots + 32 * b, 32);
  return out;
}

// TBV claim values on the device (tbv::evaluate_claims, tbv.rs:143-185).
static std::vector<Claim<F>> device_eval_claims(const Parameters<F>& P, GpuBackend& be, std::vector<Claim<F>> claims) {
  validate_claims(P.layout, claims);
  std::vector<Term<F>> terms;
  for (const Bucket& b : P.layout.buckets) {
    const auto& row = claims[b.matrix].row;
    const auto& col = claims[b.matrix].col;
    Term<F> t{b.offset, monomial_weight(b.row_offset, row.data(), row.size()) * monomial_weight(b.col_offset, col.data(), col.size()), {}};
    for (int k = 0; k < ilog2(b.cols); ++k) t.factors.push_back({F::one(), col[k]});
    for (int k = 0; k < ilog2(b.rows); ++k) t.factors.push_back({F::one(), row[k]});
    terms.push_back(std::move(t));
  }
  for (auto& c : claims) c.value = F::zero();
  // Group by lane width (terms with fewer than four factors use fewer lanes);
  // all groups go through one pass over the weights.
  std::vector<std::vector<const Term<F>*>> groups;
  std::vector<std::vector<size_t>> which;
  std::vector<size_t> group_log;
  for (size_t lanes_log = 0; lanes_log <= 4; ++lanes_log) {
    std::vector<const Term<F>*> group;
    std::vector<size_t> w;
    for (size_t i = 0; i < terms.size(); ++i)
      if (std::min<size_t>(4, terms[i].factors.size()) == lanes_log) { group.push_back(&terms[i]); w.push_back(i); }
    if (group.empty()) continue;
    groups.push_back(std::move(group));
    which.push_back(std::move(w));
    group_log.push_back(lanes_log);
  }
  auto pr = be.project_term_groups(groups, 16);
  for (size_t k = 0; k < groups.size(); ++k)
    for (size_t g = 0; g < groups[k].size(); ++g) {
      std::vector<F> low = factor_weights(groups[k][g]->factors.data(), group_log[k]);
      F v = F::zero();
      for (size_t l = 0; l < pr[k][g].size(); ++l) v += pr[k][g][l] * low[l];
      claims[P.layout.buckets[which[k][g]].matrix].value += v;
    }
  return claims;
}

void make_params(qf_params* out, const std::vector<Shape>& shapes, const Config& config) {
  // The setup commitments run on the current device when there is one; a
  // process without a device (parameter digests, statement checks) builds
  // them on the host.
  int devices = 0;
  DeviceSetup ds;
  SetupAccel<F>* accel = cudaGetDeviceCount(&devices) == cudaSuccess && devices > 0 ? &ds : nullptr;
  if (!accel) cudaGetLastError();
  out->P = std::shared_ptr<Parameters<F>>(make_parameters<F>(shapes, config, accel).release());
  out->tables = std::make_shared<DeviceTables>();
}

void info(const qf_params* params, uint64_t* active, uint64_t* logical, uint64_t* blocks, uint64_t* buckets,
          uint8_t parameter_digest[32]) {
  const auto& P = params_of(params);
  if (active) *active = P.layout.active;
  if (logical) *logical = P.layout.logical;
  if (blocks) *blocks = P.blocks();
  if (buckets) *buckets = P.layout.buckets.size();
  if (parameter_digest) std::memcpy(parameter_digest, P.pcs.parameter_digest().data(), 32);
}

void commit(const qf_params* params, const void* bva, uint64_t n_values, int bva_on_device, qf_committed* out,
            uint8_t* roots_out) {
    const auto& P = params_of(params);
    check(n_values == P.layout.active, "active BVA length mismatch");
    auto c = std::make_unique<FieldCommitted>();
    c->active = n_values;
    QF_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    auto t0 = std::chrono::steady_clock::now();
    c->bva.alloc(std::max<uint64_t>(n_values, 8));
    // The weights arrive block by block on a copy stream; block b is committed
    // as soon as its bytes have landed, so the transfer of block b + 1
    // overlaps the encoding and hashing of block b.
    const size_t live = std::min<size_t>(P.blocks(), (n_values + P.block_len - 1) / P.block_len);
    CopyPipeline copies(live);
    const cudaMemcpyKind kind = bva_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    QF_CK(cudaEventRecord(copies.begin, copies.stream));
    for (size_t b = 0; b < live; ++b) {
      const uint64_t a = uint64_t(b) * P.block_len, e = std::min<uint64_t>(a + P.block_len, n_values);
      QF_CK(cudaMemcpyAsync(c->bva.p + a, static_cast<const W*>(bva) + a, (e - a) * sizeof(W), kind, copies.stream));
      QF_CK(cudaEventRecord(copies.landed[b], copies.stream));
    }
    QF_CK(cudaEventRecord(copies.end, copies.stream));
    c->be = std::make_unique<GpuBackend>(P, c->bva.p, n_values, c->stream, static_cast<DeviceTables*>(params->tables.get()));
    for (size_t b = 0; b < P.blocks(); ++b) {
      if (b < live) QF_CK(cudaStreamWaitEvent(c->stream, copies.landed[b], 0));
      c->roots.push_back(c->be->commit_block(b));
    }
    QF_CK(cudaStreamWaitEvent(c->stream, copies.end, 0));
    QF_CK(cudaEventSynchronize(copies.end));
    float up = 0;
    QF_CK(cudaEventElapsedTime(&up, copies.begin, copies.end));
    c->upload_ms = up;
    // Padding must be zero (validate_values) — checked on the device.
    std::vector<uint64_t> seg = padding_segments(P, 0, n_values);
    if (!seg.empty()) {
      DBuf<uint64_t> dseg(seg.size());
      DBuf<unsigned int> flag(1);
      QF_CK(cudaMemcpyAsync(dseg.p, seg.data(), seg.size() * 8, cudaMemcpyHostToDevice, c->stream));
      QF_CK(cudaMemsetAsync(flag.p, 0, 4, c->stream));
      QF_LAUNCH(c->stream, "k_check_zero_segments", 0,
                k_check_zero_segments<<<unsigned(std::min<size_t>(seg.size() / 2, 148 * 8)), 256, 0, c->stream>>>(
                    reinterpret_cast<const uint8_t*>(c->bva.p), dseg.p, uint32_t(seg.size() / 2), flag.p));
      unsigned int h = 0;
      QF_CK(cudaMemcpyAsync(&h, flag.p, 4, cudaMemcpyDeviceToHost, c->stream));
      QF_CK(cudaStreamSynchronize(c->stream));
      check(h == 0, "nonzero boundary padding");
    }
    QF_CK(cudaStreamSynchronize(c->stream));
    c->commit_ms = ms_since(t0);
    if (roots_out)
      for (size_t b = 0; b < c->roots.size(); ++b) std::memcpy(roots_out + 32 * b, c->roots[b].data(), 32);
    out->state = std::move(c);
}

// HBM for resident weight blocks.  QF_RESIDENT_AUTO takes what the device
// has free now (the pool's cache included) less the proof's own peak: the EO round vectors (2.5 x
// N/stride elements) or the batch opening's tables and codewords (about 7.5 x
// packed_len elements), whichever is larger, plus the staging slots and 4 GiB.
static uint64_t resident_budget(const Parameters<F>& P, uint64_t requested) {
  if (requested != QF_RESIDENT_AUTO) return requested;
  // Blocks cached by the pool count as free: a repeated proof of the same
  // shapes finds its buffers there, and a short allocation trims the cache.
  size_t free_b = 0, total_b = 0;
  QF_CK(cudaMemGetInfo(&free_b, &total_b));
  free_b += DevicePool::cached_bytes();
  const uint64_t el = 16, m = P.pcs.packed_len(), rows = P.layout.logical >> P.config.packed_log;
  const uint64_t eo = rows * el * 5 / 2, opening = m * el * 15 / 2;
  const uint64_t need = std::max(eo, opening) + 3 * P.block_len * sizeof(W) + (uint64_t(4) << 30);
  return free_b > need ? free_b - need : 0;
}

// Recompute mode over weights that stay in host memory (`host` must outlive
// the committed handle): one streamed pass commits every block and checks
// the padding; the first `resident_bytes` worth of blocks stay in HBM.
void commit_streamed(const qf_params* params, const void* host, uint64_t n_values, uint64_t resident_bytes,
                     qf_committed* out, uint8_t* roots_out) {
  const auto& P = params_of(params);
  check(n_values == P.layout.active, "active BVA length mismatch");
  auto c = std::make_unique<FieldCommitted>();
  c->active = n_values;
  QF_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  auto t0 = std::chrono::steady_clock::now();
  const size_t resident = size_t(resident_budget(P, resident_bytes) / (P.block_len * sizeof(W)));
  c->src = std::make_unique<BlockStream>(static_cast<const W*>(host), n_values, P.block_len, resident, 3);
  c->be = std::make_unique<GpuBackend>(P, c->src.get(), c->stream, static_cast<DeviceTables*>(params->tables.get()));
  // Padding segments of every live block, relative to the block, uploaded once.
  const size_t live = c->src->live_blocks();
  std::vector<uint64_t> seg;
  std::vector<size_t> seg_at(live + 1, 0);
  for (size_t b = 0; b < live; ++b) {
    const uint64_t lo = uint64_t(b) * P.block_len;
    std::vector<uint64_t> s = padding_segments(P, lo, std::min<uint64_t>(lo + P.block_len, n_values));
    seg.insert(seg.end(), s.begin(), s.end());
    seg_at[b + 1] = seg.size();
  }
  DBuf<uint64_t> dseg(std::max<size_t>(seg.size(), 1));
  DBuf<unsigned int> flag(1);
  if (!seg.empty()) QF_CK(cudaMemcpyAsync(dseg.p, seg.data(), seg.size() * 8, cudaMemcpyHostToDevice, c->stream));
  QF_CK(cudaMemsetAsync(flag.p, 0, 4, c->stream));
  c->roots = c->be->commit_streamed([&](size_t b, const W* d, uint64_t) {
    const size_t ns = (seg_at[b + 1] - seg_at[b]) / 2;
    if (!ns) return;
    QF_LAUNCH(c->stream, "k_check_zero_segments", 0,
              k_check_zero_segments<<<unsigned(std::min<size_t>(ns, 148 * 8)), 256, 0, c->stream>>>(
                  reinterpret_cast<const uint8_t*>(d), dseg.p + seg_at[b], uint32_t(ns), flag.p));
  });
  unsigned int h = 0;
  QF_CK(cudaMemcpyAsync(&h, flag.p, 4, cudaMemcpyDeviceToHost, c->stream));
  QF_CK(cudaStreamSynchronize(c->stream));
  check(h == 0, "nonzero boundary padding");
  c->commit_ms = ms_since(t0);
  c->upload_ms = 0;
  if (roots_out)
    for (size_t b = 0; b < c->roots.size(); ++b) std::memcpy(roots_out + 32 * b, c->roots[b].data(), 32);
  out->state = std::move(c);
}

std::string statement_json(const qf_params* params, const uint8_t* roots) {
  return commitment_json(make_statement(params_of(params), roots_from(params, roots)));
}

std::vector<uint8_t> benchmark_points_bytes(const qf_params* params, const uint8_t* roots) {
  auto pts = benchmark_points<F>(make_statement(params_of(params), roots_from(params, roots)));
  ByteWriter w;
  for (const auto& [r, c] : pts) {
    for (const F& v : r) w.field(v);
    for (const F& v : c) w.field(v);
  }
  return std::move(w.out);
}

std::vector<uint8_t> eval_claims(const qf_params* params, const qf_committed* committed, const uint8_t* points, size_t len) {
  const auto* fc = static_cast<const FieldCommitted*>(committed->state.get());
  auto cl = parse_claims(params_of(params), points, len, false);
  return write_claims(device_eval_claims(params_of(params), *fc->be, std::move(cl)), true);
}

std::vector<uint8_t> prove(const qf_params* params, qf_committed* committed, const uint8_t* claims, size_t claims_len,
                           qf_profile* profile) {
    auto* fc = static_cast<FieldCommitted*>(committed->state.get());
    const auto& P = params_of(params);
    auto cl = parse_claims(P, claims, claims_len, true);
    auto t0 = std::chrono::steady_clock::now();
    Commitment st = make_statement(P, fc->roots);
    Transcript<F> t = statement_transcript(P, st, cl);
    Query<F> q = compile(P.layout, cl, t);
    auto [eo, term] = eo_prove<F>(*fc->be, P.layout.logical, size_t(1) << P.config.packed_log, q, t);
    double eo_ms = ms_since(t0);
    std::vector<uint8_t> ctx = opening_context<F>(t.state, 0);
    BatchOpening<F> op = fc->roots.size() > 1 ? open_batch(P.pcs, *fc->be, fc->roots, term.point_msb, ctx)
                                                    : open_single(P.pcs, *fc->be, fc->roots[0], term.point_msb, ctx);
    fc->be->release_opening_state();
    check(op.claimed_value * term.scale == term.value, "QAFold/EO terminal mismatch");
    Proof<F> pr;
    pr.eo = std::move(eo);
    pr.opening_value = op.claimed_value;
    pr.opening_proof = std::move(op.wire);
    std::vector<uint8_t> bytes = proof_to_bytes(pr);
    if (profile) {
      profile->commit_ms = fc->commit_ms;
      profile->upload_ms = fc->upload_ms;
      profile->eo_ms = eo_ms;
      profile->projection_ms = op.times.projection_ms;
      profile->folding_ms = op.times.folding_ms;
      profile->sumcheck_ms = op.times.sumcheck_ms;
      profile->binding_ms = op.times.binding_ms;
      profile->native_opening_ms = op.times.native_opening_ms;
      profile->decide_ms = op.times.decide_ms;
      profile->open_ms = ms_since(t0);
      profile->kernel_launches = qfg::KernelClock::launches.load();
    }
    return bytes;
}

void verify(const qf_params* params, const uint8_t* roots, const uint8_t* claims, size_t claims_len, const uint8_t* proof,
            size_t proof_len) {
    const auto& P = params_of(params);
    auto cl = parse_claims(P, claims, claims_len, true);
    Proof<F> pr = proof_from_bytes<F>(proof, proof_len);
    verify_proof(P, make_statement(P, roots_from(params, roots)), cl, pr);
}


void stream_info(const qf_committed* committed, uint64_t* h2d_bytes, uint64_t* resident_blocks, uint64_t* live_blocks) {
  const auto* fc = static_cast<const FieldCommitted*>(committed->state.get());
  if (h2d_bytes) *h2d_bytes = fc->src ? fc->src->h2d_bytes() : 0;
  if (resident_blocks) *resident_blocks = fc->src ? fc->src->resident_blocks() : 0;
  if (live_blocks) *live_blocks = fc->src ? fc->src->live_blocks() : 0;
}

// One rank's device work in a block-sharded proof: a GPU backend over a copy
// of the BVA that holds only this rank's blocks (zero elsewhere), so every
// weight-linear sum it returns is the rank's part.
class GpuShard final : public ShardBackend<F> {
 public:
  explicit GpuShard(GpuBackend& be) : be_(be) {}
  Digest commit_block(size_t b) override { return be_.commit_block(b); }
  std::vector<std::vector<F>> project_blocks(const std::vector<F>& outer, size_t blocks) override {
    return be_.project_blocks(outer, blocks);
  }
  void apply_images(const std::vector<F>& images) override { be_.apply_images(images); }
  std::vector<F> fold_part(const std::vector<F>& fold_weights) override { return be_.fold_values(fold_weights); }
  Digest commit_folded(std::vector<F> values) override { return be_.commit_folded_values(values); }
  void sumcheck_message(F m[2]) override { be_.sumcheck_message(m); }
  void sumcheck_fold(F ch) override { be_.sumcheck_fold(ch); }
  F sumcheck_final_value() override { return be_.sumcheck_final_value(); }
  F sumcheck_final_weight() override { return be_.sumcheck_final_weight(); }
  void write_block_rows(ByteWriter& w, size_t b, const RowSelection& sel, const Digest& root) override {
    be_.write_block_rows(w, b, sel, root);
  }
  void write_folded_rows(ByteWriter& w, const RowSelection& sel) override { be_.write_folded_rows(w, sel); }
  const CodewordView<F>& folded_codeword() override { return be_.folded_codeword(); }
  std::vector<F> folded_opening(const std::vector<F>& point, size_t col_log, std::vector<F>& rw) override {
    return be_.folded_opening(point, col_log, rw);
  }
  TopRoundAccel<F>* top_round_accel() override { return be_.top_round_accel(); }
  DecideAccel<F>* decide_accel() override { return be_.decide_accel(); }
  void cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) override {
    be_.cross_terms(q, stride, pos, neg);
  }
  F eo_build(const Query<F>& q, F ch, F inv, size_t logical, size_t stride) override {
    return be_.eo_build(q, ch, inv, logical, stride);
  }
  std::array<F, 2> eo_round_cross() override { return be_.eo_round_cross(); }
  void eo_round_fold(F inv, F ch) override { be_.eo_round_fold(inv, ch); }
  std::array<F, 2> eo_terminal() override { return be_.eo_terminal(); }

 private:
  GpuBackend& be_;
};

// Whether any zero-padding entry in [lo, hi) of the device BVA is nonzero.
static bool padding_nonzero(const Parameters<F>& P, const W* d_bva, uint64_t lo, uint64_t hi, cudaStream_t s) {
  const std::vector<uint64_t> seg = padding_segments(P, lo, hi);
  if (seg.empty()) return false;
  DBuf<uint64_t> dseg(seg.size());
  DBuf<unsigned int> flag(1);
  QF_CK(cudaMemcpyAsync(dseg.p, seg.data(), seg.size() * 8, cudaMemcpyHostToDevice, s));
  QF_CK(cudaMemsetAsync(flag.p, 0, 4, s));
  QF_LAUNCH(s, "k_check_zero_segments", 0,
            k_check_zero_segments<<<unsigned(std::min<size_t>(seg.size() / 2, 148 * 8)), 256, 0, s>>>(
                reinterpret_cast<const uint8_t*>(d_bva + lo), dseg.p, uint32_t(seg.size() / 2), flag.p));
  unsigned int h = 0;
  QF_CK(cudaMemcpyAsync(&h, flag.p, 4, cudaMemcpyDeviceToHost, s));
  QF_CK(cudaStreamSynchronize(s));
  return h != 0;
}

// A rank of a block-sharded proof: its blocks of the host BVA copied to the
// current device (the rest of the copy zero), the padding of its range
// checked (the flags summed over the ranks, so all stop together), its
// blocks committed and the roots gathered, the claims given or summed from
// every rank's part, then the outer prover over the sharding layer.
std::vector<uint8_t> prove_sharded(const qf_params* params, const void* host_bva, uint64_t n_values, int rank, int world,
                                   qf_gather_fn gather, qf_reduce_fn reduce, void* ctx, const uint8_t* claims,
                                   size_t claims_len, uint8_t* roots_out) {
  const auto& P = params_of(params);
  check(n_values == P.layout.active, "active BVA length mismatch");
  CallbackComm comm(rank, world, gather, ctx, reduce);
  const BlockShards shards(P.blocks(), world);
  struct Stream {
    cudaStream_t s = nullptr;
    ~Stream() { if (s) cudaStreamDestroy(s); }
  } st;
  QF_CK(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
  DBuf<W> bva(std::max<uint64_t>(n_values, 8));
  QF_CK(cudaMemsetAsync(bva.p, 0, bva.n * sizeof(W), st.s));
  const uint64_t lo = std::min<uint64_t>(n_values, uint64_t(shards.first(rank)) * P.block_len);
  const uint64_t hi = std::min<uint64_t>(n_values, uint64_t(shards.first(rank + 1)) * P.block_len);
  if (hi > lo)
    QF_CK(cudaMemcpyAsync(bva.p + lo, static_cast<const W*>(host_bva) + lo, (hi - lo) * sizeof(W), cudaMemcpyHostToDevice,
                          st.s));
  uint64_t bad = padding_nonzero(P, bva.p, lo, hi, st.s) ? 1 : 0;
  comm.all_reduce_sum(&bad, 1);
  check(bad == 0, "nonzero boundary padding");
  std::vector<uint8_t> wire;
  {
    GpuBackend be(P, bva.p, n_values, st.s, static_cast<DeviceTables*>(params->tables.get()));
    GpuShard shard(be);
    ShardedBackend<F> sharded(P, shard, comm);
    const std::vector<Digest> roots = sharded.commit_all();
    std::vector<Claim<F>> cl;
    if (claims) {
      cl = parse_claims(P, claims, claims_len, true);
    } else {
      std::vector<Claim<F>> pts;
      for (const auto& [r, c] : benchmark_points<F>(make_statement(P, roots))) pts.push_back({r, c, F::zero()});
      cl = sum_claims(comm, device_eval_claims(P, be, std::move(pts)));
    }
    wire = qf::prove_sharded(P, sharded, roots, cl);
    if (roots_out)
      for (size_t b = 0; b < roots.size(); ++b) std::memcpy(roots_out + 32 * b, roots[b].data(), 32);
    QF_CK(cudaStreamSynchronize(st.s));  // the backend's buffers go back to the pool next
  }
  return wire;
}

}  // namespace

// LogUp range audit: alpha from the seed, the weights' fraction sum on the
// device, the table side from the multiplicities.
void range_audit(const qf_params* params, const qf_committed* committed, const uint8_t seed[32], uint64_t* mult_out,
                 size_t n_bins, uint8_t alpha_out[16], uint8_t lhs_out[16], uint8_t rhs_out[16], int* holds) {
  const auto* fc = static_cast<const FieldCommitted*>(committed->state.get());
  check(!mult_out || n_bins == RangeTable<W>::kBins, "range audit: multiplicities need 256 (int8) or 65536 (int16) bins");
  const F alpha = range_audit_alpha<F>(seed);
  std::vector<uint64_t> mult;
  const std::array<F, 2> frac = fc->be->range_audit(alpha, mult);
  const F lhs = frac[0] * frac[1].inverse();
  const F rhs = logup_table_sum<F, W>(alpha, mult);
  uint64_t total = 0;
  for (uint64_t m : mult) total += m;
  if (mult_out) std::memcpy(mult_out, mult.data(), mult.size() * 8);
  if (alpha_out) alpha.to_bytes(alpha_out);
  if (lhs_out) lhs.to_bytes(lhs_out);
  if (rhs_out) rhs.to_bytes(rhs_out);
  if (holds) *holds = (lhs == rhs && total == fc->active) ? 1 : 0;
}

const qfc::FieldApi kFieldApi = {sizeof(W),  make_params, info,   commit,      commit_streamed,
                                 statement_json, benchmark_points_bytes, eval_claims, prove, verify,
                                 stream_info, prove_sharded, range_audit};

}  // namespace QFB_NS
