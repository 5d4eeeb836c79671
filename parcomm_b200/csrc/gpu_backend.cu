// CUDA backend for the packed PCS and EO of one field (see gpu_backend.cuh).
#include "gpu_backend.cuh"
#include "kernels/commit.cuh"
#include "kernels/open.cuh"
#include "kernels/vec.cuh"
#include "kernels/audit.cuh"
#include "kernels/dot_mma.cuh"
#if !defined(QF_FIELD_KB)
#include "kernels/imma_f65521.cuh"
#endif
#include "intops.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <set>

namespace QFB_NS {

static constexpr int kThreads = 256;
// Folding rounds over vectors of at most this many elements (LiteBullet,
// sumcheck, EO binary rounds) run on the host: each device round costs a
// launch and a synchronisation (about 20 us), more than the host's 2n
// extension products at this length.
static constexpr uint64_t kHostTail = 512;
// Operation counts of this field's arithmetic, for the integer roofline.
#if defined(QF_FIELD_KB)
static constexpr const qf_intops::FieldOps& kOps = qf_intops::kKoalaBear;
#else
static constexpr const qf_intops::FieldOps& kOps = qf_intops::kF65521;
#endif

// The exact integer-limb tensor-core kernels exist for F65521^8 (8-bit
// weights); KoalaBear keeps its 64-bit IMAD kernels.
static bool imma_on() {
#if defined(QF_FIELD_KB)
  return false;
#else
  return KernelOptions::imma.load() != 0;
#endif
}
// The extension-product sums of the EO, sumcheck and LiteBullet rounds:
// on the tensor cores (kernels/dot_mma.cuh) where that measured faster on
// B200 in the 8B-shape step, on the CUDA cores elsewhere (core_dots 0);
// core_dots 1 takes the CUDA cores everywhere, 2 the tensor cores
// everywhere.  The tensor-core sums win on the long vectors: EO dot and
// first cross pair 2.5x / 2.2x, EO query fold 1.4x / 1.13x, sumcheck message
// 1.7x / 1.3x and fold 1.09x / 1.19x (F65521 / KoalaBear).  On the short
// vectors of the LiteBullet rounds and the small EO rounds the chunked warp
// loop and its staging cost more than they save (0.7x - 0.9x), except the
// KoalaBear LiteBullet cross pair (1.03x).
enum class Dots { kEoDotCross, kEoFoldQueryCross, kEoFoldCross, kSumMessage, kSumFold, kLbCross, kLbFold, kDot };
static bool tc_dots(Dots k) {
  const int opt = KernelOptions::core_dots.load();
  if (opt != 0) return opt == 2;
#if defined(QF_FIELD_KB)
  return k == Dots::kEoDotCross || k == Dots::kEoFoldQueryCross || k == Dots::kSumMessage || k == Dots::kSumFold ||
         k == Dots::kLbCross;
#else
  return k == Dots::kEoDotCross || k == Dots::kEoFoldQueryCross || k == Dots::kSumMessage || k == Dots::kSumFold;
#endif
}
// Grid of the persistent tensor-core weight kernels: four CTAs per SM.
static unsigned mma_grid() {
  static const int sms = [] {
    int d = 0, n = 148;
    if (cudaGetDevice(&d) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess) n = 148;
    return n;
  }();
  return unsigned(sms * 4);
}
// Grid of a tensor-core product kernel over `count` indices (one per thread
// and chunk), at most four CTAs per SM.
static unsigned dot_grid(uint64_t count) {
  return unsigned(std::max<uint64_t>(1, std::min<uint64_t>((count + qfd::kDotThreads - 1) / qfd::kDotThreads, mma_grid())));
}

template <class K>
static void set_smem(K kernel, size_t bytes) {
  QF_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}

// ---------------------------------------------------------------- codeword view
std::vector<F> DeviceCodeword::fold_rows(size_t n_rows, const std::vector<F>& w) const {
  DBuf<Fe> dw(n_cols), out(n_rows);
  QF_CK(cudaMemcpyAsync(dw.p, w.data(), n_cols * 16, cudaMemcpyHostToDevice, stream));
  QF_LAUNCH(stream, "k_row_fold", uint64_t(n_rows) * n_cols * 16 + uint64_t(n_rows) * 16, qfd::k_row_fold<<<grid_for(n_rows, kThreads), kThreads, 0, stream>>>(cw.p, n_ext, n_rows, int(n_cols), dw.p, out.p));
  std::vector<F> h(n_rows);
  QF_CK(cudaMemcpyAsync(h.data(), out.p, n_rows * 16, cudaMemcpyDeviceToHost, stream));
  QF_CK(cudaStreamSynchronize(stream));
  return h;
}

std::vector<F> DeviceCodeword::project_rows(size_t n_rows, const std::vector<F>& w) const {
  // The row weights arrive as a full table; upload it as the low table of a
  // single-entry two-level product.
  DBuf<Fe> lo(n_rows), hi(1);
  F one = F::one();
  QF_CK(cudaMemcpyAsync(lo.p, w.data(), n_rows * 16, cudaMemcpyHostToDevice, stream));
  QF_CK(cudaMemcpyAsync(hi.p, &one, 16, cudaMemcpyHostToDevice, stream));
  const int chunks = int(std::min<size_t>(64, (n_rows + kThreads - 1) / kThreads));
  DBuf<Fe> part(n_cols * chunks);
  dim3 grid(chunks, unsigned(n_cols));
  QF_LAUNCH(stream, "k_row_project", uint64_t(n_rows) * n_cols * 16 + uint64_t(n_rows) * 16, qfd::k_row_project<<<grid, kThreads, 0, stream>>>(cw.p, n_ext, n_rows, hi.p, lo.p, ilog2(n_rows), part.p));
  std::vector<F> hp(n_cols * chunks);
  QF_CK(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 16, cudaMemcpyDeviceToHost, stream));
  QF_CK(cudaStreamSynchronize(stream));
  std::vector<F> out(n_cols, F::zero());
  for (size_t c = 0; c < n_cols; ++c)
    for (int k = 0; k < chunks; ++k) out[c] += hp[c * chunks + k];
  return out;
}

std::vector<std::vector<F>> DeviceCodeword::rows(const std::vector<size_t>& idx) const {
  std::vector<std::vector<F>> out;
  if (idx.empty()) return out;
  std::vector<uint64_t> id(idx.begin(), idx.end());
  DBuf<uint64_t> did(id.size());
  DBuf<Fe> dout(id.size() * n_cols);
  QF_CK(cudaMemcpyAsync(did.p, id.data(), id.size() * 8, cudaMemcpyHostToDevice, stream));
  QF_LAUNCH(stream, "k_gather_rows", uint64_t(id.size()) * n_cols * 32, qfd::k_gather_rows<<<grid_for(id.size() * n_cols, kThreads, 1 << 20), kThreads, 0, stream>>>(cw.p, n_ext, int(n_cols), did.p,
                                                                                               uint32_t(id.size()), dout.p));
  std::vector<F> h(id.size() * n_cols);
  QF_CK(cudaMemcpyAsync(h.data(), dout.p, h.size() * 16, cudaMemcpyDeviceToHost, stream));
  QF_CK(cudaStreamSynchronize(stream));
  for (size_t q = 0; q < id.size(); ++q) out.emplace_back(h.begin() + q * n_cols, h.begin() + (q + 1) * n_cols);
  return out;
}

std::vector<std::vector<Digest>> DeviceCodeword::paths(const std::vector<size_t>& idx) const {
  std::vector<std::vector<Digest>> out;
  if (idx.empty()) return out;
  const int depth = ilog2(n_ext);
  std::vector<uint64_t> id(idx.begin(), idx.end());
  DBuf<uint64_t> did(id.size()), doff(level_off.size());
  DBuf<uint4> dout(id.size() * depth * 2);
  QF_CK(cudaMemcpyAsync(did.p, id.data(), id.size() * 8, cudaMemcpyHostToDevice, stream));
  QF_CK(cudaMemcpyAsync(doff.p, level_off.data(), level_off.size() * 8, cudaMemcpyHostToDevice, stream));
  if (depth > 0) {
    QF_LAUNCH(stream, "k_gather_paths", uint64_t(id.size()) * depth * 64, qfd::k_gather_paths<<<grid_for(id.size() * depth, kThreads, 1 << 20), kThreads, 0, stream>>>(tree.p, doff.p, depth, did.p,
                                                                                                 uint32_t(id.size()), dout.p));
  }
  std::vector<uint4> h(id.size() * depth * 2);
  QF_CK(cudaMemcpyAsync(h.data(), dout.p, h.size() * 16, cudaMemcpyDeviceToHost, stream));
  QF_CK(cudaStreamSynchronize(stream));
  for (size_t q = 0; q < id.size(); ++q) {
    std::vector<Digest> p;
    for (int l = 0; l < depth; ++l) p.push_back(digest_from_words(&h[(q * depth + l) * 2]));
    out.push_back(std::move(p));
  }
  return out;
}

std::vector<F> DeviceCodeword::entries() const {
  std::vector<F> h(n_ext * n_cols);
  QF_CK(cudaMemcpyAsync(h.data(), cw.p, h.size() * 16, cudaMemcpyDeviceToHost, stream));
  QF_CK(cudaStreamSynchronize(stream));
  return h;
}

// Planar tile kernels take up to 2^kMaxTileLog elements (128 KiB of shared
// memory); the opt-in is set once per device.
static void configure_tile_kernels() {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  QF_CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return;
  const size_t bytes = qfd::kTileSmem;
  set_smem(qfd::k_pack_mobius_tile, bytes);
  set_smem(qfd::k_copy_mobius_tile, bytes);
  set_smem(qfd::k_wht_tile<false>, bytes);
  set_smem(qfd::k_wht_tile<true>, bytes);
  set_smem(qfd::k_butterfly_strided<qfd::kMobius>, bytes);
  set_smem(qfd::k_butterfly_strided<qfd::kWht>, bytes);
  set_smem(qfd::k_mobius_wht_strided, bytes + qfd::kPrefetchSmem);
  set_smem(qfd::k_wht_alpha_wht_tile, bytes + qfd::kAlphaStageSmem);
#if !defined(QF_FIELD_KB)
  // 38 KiB of static shared memory plus the 32 KiB weight double buffer.
  set_smem(qfd::k_eq_project_blocks, qfd::kEqWeightSmem);
#endif
  done.insert(dev);
}

// ---------------------------------------------------------------- backend
GpuBackend::GpuBackend(const Parameters<F>& p, const W* d_bva, size_t active, cudaStream_t s, DeviceTables* tables)
    : P_(p), bva_(d_bva), active_(active), s_(s), tables_(tables ? tables : &own_tables_) {
  configure_tile_kernels();
  partials_.alloc(qfd::kRedHeader + 148 * 8 * 3);
  QF_CK(cudaMemsetAsync(partials_.p, 0, 16, s_));  // the reduction counter starts at zero
}
GpuBackend::GpuBackend(const Parameters<F>& p, BlockStream* src, cudaStream_t s, DeviceTables* tables)
    : P_(p), bva_(nullptr), src_(src), active_(src->active()), s_(s), tables_(tables ? tables : &own_tables_) {
  configure_tile_kernels();
  check(src->block_len() == P_.block_len, "block length of the weight stream");
  if (src->on_device()) bva_ = src->host();  // gathers read the resident weights directly
  partials_.alloc(qfd::kRedHeader + 148 * 8 * 3);
  QF_CK(cudaMemsetAsync(partials_.p, 0, 16, s_));  // the reduction counter starts at zero
}
GpuBackend::~GpuBackend() {}

void GpuBackend::release_opening_state() {
  QF_CK(cudaStreamSynchronize(s_));
  for (DBuf<Fe>* b : {&weights_, &values_, &tmp_v_, &tmp_w_, &wit_, &qv_, &wit2_, &qv2_, &rw_d_}) b->reset();
  folded_.reset();
  scratch_.reset();
  single_cw_ = nullptr;
  open_cw_ = nullptr;
  sum_len_ = 0;
  eo_len_ = 0;
  msg_valid_ = false;
  host_v_.clear();
  host_w_.clear();
  host_wit_.clear();
  host_qv_.clear();
}

// ---------------------------------------------------------------- streamed weights
BlockStream::BlockStream(const W* host, uint64_t active, uint64_t block_len, size_t resident, int slots)
    : host_(host), active_(active), block_len_(block_len) {
  check(slots >= 2, "at least two staging slots");
  live_ = size_t((active + block_len - 1) / block_len);
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, host) == cudaSuccess && attr.type == cudaMemoryTypeDevice) {
    device_ = true;
    resident_ = live_;
    return;
  }
  cudaGetLastError();
  resident_ = std::min(resident, live_);
  if (resident_) resident_buf_.alloc(resident_ * block_len);
  const size_t streamed = live_ - resident_;
  slot_buf_.resize(std::min<size_t>(size_t(slots), streamed));
  for (auto& b : slot_buf_) b.alloc(block_len);
  slot_block_.assign(slot_buf_.size(), ~size_t(0));
  QF_CK(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
  landed_.assign(live_, nullptr);
  for (auto& e : landed_) QF_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  freed_.assign(slot_buf_.size(), nullptr);
  for (auto& e : freed_) QF_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}
BlockStream::~BlockStream() {
  if (copy_) cudaStreamSynchronize(copy_);
  for (auto& e : landed_)
    if (e) cudaEventDestroy(e);
  for (auto& e : freed_)
    if (e) cudaEventDestroy(e);
  if (copy_) cudaStreamDestroy(copy_);
}

void BlockStream::for_each(cudaStream_t s, const BlockFn& fn) {
  if (device_) {
    for (size_t i = 0; i < live_; ++i)
      fn(i, host_ + uint64_t(i) * block_len_, std::min<uint64_t>(block_len_, active_ - uint64_t(i) * block_len_));
    return;
  }
  const size_t K = slot_buf_.size();
  auto n_of = [&](size_t b) { return std::min<uint64_t>(block_len_, active_ - uint64_t(b) * block_len_); };
  // Visiting order.  The first pass goes in ascending order (it also copies
  // the resident blocks).  Later passes start with the streamed blocks the
  // previous pass left in the staging slots (no copy), then spread the other
  // streamed blocks evenly among the resident ones, so that their copies
  // overlap the resident blocks' launches.
  std::vector<size_t> order;
  if (!resident_ready_ || K == 0) {
    for (size_t t = 0; t < live_; ++t) order.push_back(t);
  } else {
    std::vector<bool> staged(live_, false);
    for (size_t k = 0; k < K; ++k)
      if (slot_block_[k] < live_ && slot_block_[k] >= resident_ && !staged[slot_block_[k]]) {
        staged[slot_block_[k]] = true;
        order.push_back(slot_block_[k]);
      }
    std::vector<size_t> rest;
    for (size_t b = resident_; b < live_; ++b)
      if (!staged[b]) rest.push_back(b);
    const size_t ns = rest.size(), nr = resident_;
    for (size_t q = 0, a = 0, r = 0; q < ns + nr; ++q) {
      if (a < ns && (r >= nr || a * (ns + nr) <= q * ns)) order.push_back(rest[a++]);
      else order.push_back(r++);
    }
  }
  // The t-th streamed block of the pass takes slot cycle[t % K]: the first K
  // keep the slots that already hold them, the others take the free slots;
  // ps[p] counts the streamed blocks before visiting position p.
  std::vector<size_t> ps(live_ + 1, 0), streamed;
  for (size_t p = 0; p < live_; ++p) {
    ps[p + 1] = ps[p] + (order[p] >= resident_ ? 1 : 0);
    if (order[p] >= resident_) streamed.push_back(order[p]);
  }
  std::vector<int> cycle(K, -1), slot_of(live_, -1);
  std::vector<bool> taken(K, false);
  for (size_t t = 0; t < std::min(K, streamed.size()); ++t)
    for (size_t k = 0; k < K; ++k)
      if (!taken[k] && slot_block_[k] == streamed[t]) { cycle[t] = int(k); taken[k] = true; break; }
  for (size_t t = 0; t < K; ++t)
    for (size_t k = 0; cycle[t] < 0 && k < K; ++k)
      if (!taken[k]) { cycle[t] = int(k); taken[k] = true; }
  for (size_t t = 0; t < streamed.size(); ++t) slot_of[streamed[t]] = cycle[t % K];
  auto dev_of = [&](size_t b) -> W* {
    return b < resident_ ? resident_buf_.p + uint64_t(b) * block_len_ : slot_buf_[size_t(slot_of[b])].p;
  };
  // A slot's new copy waits until the launches on its previous block are
  // done (freed_); a block still staged from the previous pass is not copied.
  auto issue = [&](size_t b) {
    if (b < resident_ && resident_ready_) return;
    if (b >= resident_) {
      const size_t k = size_t(slot_of[b]);
      if (slot_block_[k] == b) return;
      QF_CK(cudaStreamWaitEvent(copy_, freed_[k], 0));
      slot_block_[k] = b;
    }
    const uint64_t n = n_of(b);
    QF_CK(cudaMemcpyAsync(dev_of(b), host_ + uint64_t(b) * block_len_, n * sizeof(W), cudaMemcpyHostToDevice, copy_));
    QF_CK(cudaEventRecord(landed_[b], copy_));
    copied_ += n * sizeof(W);
  };
  // Streamed copies run up to K streamed blocks ahead of the compute
  // position (so a slot is reused only after its previous block's launches
  // were enqueued); on the first pass the resident ones up to K positions.
  const size_t ahead = std::max<size_t>(K, 1);
  size_t issued = 0;
  for (size_t i = 0; i < live_; ++i) {
    while (issued < live_) {
      const size_t b = order[issued];
      if (b >= resident_ ? ps[issued] >= ps[i] + K : (!resident_ready_ && issued >= i + ahead)) break;
      issue(b);
      ++issued;
    }
    const size_t b = order[i];
    if (!(b < resident_ && resident_ready_)) QF_CK(cudaStreamWaitEvent(s, landed_[b], 0));
    fn(b, dev_of(b), n_of(b));
    if (b >= resident_) QF_CK(cudaEventRecord(freed_[size_t(slot_of[b])], s));
  }
  if (resident_) resident_ready_ = true;
}

const Fe* DeviceTables::alpha(const PcsParams<F>& pp, size_t level, int which) {
  int dev = 0;
  QF_CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu_);
  auto key = std::make_tuple(dev, level, which);
  auto it = bufs_.find(key);
  if (it == bufs_.end()) {
    const auto& a = pp.seq.codes.at(level).alphas.at(size_t(which));
    DBuf<Fe> b(a.size());
    // A copy from pageable memory may return before its DMA has landed, and
    // the readers run on non-blocking streams: wait for the legacy stream.
    QF_CK(cudaMemcpy(b.p, a.data(), a.size() * 16, cudaMemcpyHostToDevice));
    QF_CK(cudaStreamSynchronize(0));
    it = bufs_.emplace(key, std::move(b)).first;
  }
  return it->second.p;
}

// Grid of a persistent tile kernel: at most one CTA per SM (a CTA's 128 KiB of
// tile planes leaves room for one), each looping over its tiles.
static unsigned tile_grid(uint64_t n_tiles) {
  static const int sms = [] {
    int d = 0, n = 148;
    if (cudaGetDevice(&d) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess) n = 148;
    return n;
  }();
  return unsigned(std::min<uint64_t>(n_tiles, uint64_t(sms)));
}

// The first min(12, logR) WHT levels of a 2^logm-entry half, optionally
// multiplying by alpha first (a CTA size per variant).
static void wht_tile_launch(cudaStream_t s, const Fe* src, Fe* dst, const Fe* alpha, int logR, int logm, int wl) {
  check(logm <= 30, "transform passes index a codeword of at most 2^31 elements");
  const uint32_t tiles = uint32_t(size_t(1) << (logm - wl));
  if (alpha)
    qfd::k_wht_tile<true><<<tile_grid(tiles), qfd::kAlphaTileThreads, qfd::kTileSmem, s>>>(src, dst, alpha, logR, wl, tiles);
  else
    qfd::k_wht_tile<false><<<tile_grid(tiles), qfd::kTileThreads, qfd::kTileSmem, s>>>(src, dst, nullptr, logR, wl, tiles);
}

// 2^cb consecutive group bases per tile of a k-level strided pass: 64-byte
// runs at k = 10, the full 4096-element tile below that.
static int strided_cb(int k, int logm) { return std::min(k >= 10 ? 2 : qfd::kMaxTileLog - k, logm - k); }

// ---------------------------------------------------------------- pass autotuner
// How many levels each strided pass takes is a choice: one deep pass is
// issue-bound (its middle stages run on the ALU and shared memory), a shallow
// one runs near copy speed but adds a pass over HBM.  The tuner times one
// pass of every depth k = 1..10 of each transform once per process, on a
// 2^24-element proxy half (256 MiB, past L2) with the access pattern of the
// real passes, and splits a span of levels into the cheapest sequence of
// depths (dynamic programming over the measured costs).  Any split gives the
// same bytes.  QF_TUNE=0 keeps the greedy split (depth 10, then the rest).
namespace {
struct PassTuner {
  std::mutex mu;
  std::atomic<bool> ready{false};
  float ms[2][11] = {};  // [op][k]: one pass over the proxy
  std::map<std::pair<int, int>, std::vector<int>> plans;  // (op, span) -> depths

  static bool enabled() {
    const char* e = std::getenv("QF_TUNE");
    return !(e && e[0] == '0');
  }

  template <int OP>
  float time_pass(cudaStream_t s, Fe* buf, int k) {
    constexpr int kLogm = 24, kLo = 12;
    const int cb = strided_cb(k, kLogm);
    const uint32_t tiles = uint32_t(uint64_t(1) << (kLogm - k - cb));
    cudaEvent_t a, b;
    QF_CK(cudaEventCreate(&a));
    QF_CK(cudaEventCreate(&b));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      QF_CK(cudaEventRecord(a, s));
      qfd::k_butterfly_strided<OP><<<tile_grid(tiles), qfd::kTileThreads, qfd::kTileSmem, s>>>(buf, buf, kLogm, kLo, k, cb,
                                                                                                  tiles);
      QF_CK(cudaGetLastError());
      QF_CK(cudaEventRecord(b, s));
      QF_CK(cudaEventSynchronize(b));
      float t = 0;
      QF_CK(cudaEventElapsedTime(&t, a, b));
      if (rep) best = std::min(best, t);  // the first run warms up
    }
    QF_CK(cudaEventDestroy(a));
    QF_CK(cudaEventDestroy(b));
    return best;
  }

  void tune(cudaStream_t s) {
    std::lock_guard<std::mutex> g(mu);
    if (ready) return;
    DBuf<Fe> buf(size_t(1) << 24);
    QF_CK(cudaMemsetAsync(buf.p, 0, (size_t(1) << 24) * 16, s));
    std::string note;
    for (int k = 1; k <= 10; ++k) {
      ms[qfd::kMobius][k] = time_pass<qfd::kMobius>(s, buf.p, k);
      ms[qfd::kWht][k] = time_pass<qfd::kWht>(s, buf.p, k);
      char b[96];
      std::snprintf(b, sizeof b, "%s\"%d\":[%.4f,%.4f]", k > 1 ? "," : "", k, ms[qfd::kMobius][k], ms[qfd::kWht][k]);
      note += b;
    }
    KernelClock::note("strided_pass_ms_per_2^24_mobius_wht", "{" + note + "}");
    ready = true;
  }

  // Depths for `span` levels: measured optimum, or greedy before tuning.
  std::vector<int> plan(int op, int span) {
    std::vector<int> greedy;
    for (int left = span; left > 0; left -= std::min(10, left)) greedy.push_back(std::min(10, left));
    if (!ready) return greedy;
    std::lock_guard<std::mutex> g(mu);
    auto key = std::make_pair(op, span);
    auto it = plans.find(key);
    if (it != plans.end()) return it->second;
    std::vector<float> best(span + 1, 1e30f);
    std::vector<int> pick(span + 1, 0);
    best[0] = 0;
    for (int s = 1; s <= span; ++s)
      for (int k = 1; k <= std::min(10, s); ++k)
        if (best[s - k] + ms[op][k] < best[s]) { best[s] = best[s - k] + ms[op][k]; pick[s] = k; }
    std::vector<int> out;
    for (int s = span; s > 0; s -= pick[s]) out.push_back(pick[s]);
    std::string desc;
    for (int k : out) desc += (desc.empty() ? "" : "+") + std::to_string(k);
    KernelClock::note(std::string(op == qfd::kMobius ? "plan_mobius_" : "plan_wht_") + std::to_string(span), "\"" + desc + "\"");
    return plans.emplace(key, out).first->second;
  }
};
PassTuner g_tuner;
}  // namespace

// One launch, recorded by the kernel clock (timed) or plain (the
// allocation-free path).
template <class Fn>
static void launch(cudaStream_t s, bool timed, const char* name, uint64_t bytes, uint64_t ops, Fn&& fn) {
  if (timed) {
    QF_LAUNCH_OPS(s, name, bytes, ops, fn());
  } else {
    fn();
    QF_CK(cudaGetLastError());
  }
}

// Butterfly levels [from, to) over a half of 2^logm entries, in strided
// passes of at most 10 levels (the tuner's split).  The first pass reads
// `src` and writes `dst`; the others work in place on `dst` (src == dst: all
// in place).  `to` is at most logR for the per-column WHT and logm for the
// Mobius transform of the whole message.  `allow_tuning` is false on the
// allocation-free path.
template <int OP>
static void strided_passes(cudaStream_t s, const Fe* src, Fe* dst, int logR, int logm, int from, int to, bool timed = true,
                           bool allow_tuning = true) {
  if (to <= from) return;
  check(logm <= 30, "transform passes index a codeword of at most 2^31 elements");
  if (allow_tuning && PassTuner::enabled() && !g_tuner.ready) g_tuner.tune(s);
  int lo = from;
  for (int k : g_tuner.plan(OP, to - from)) {
    const int cb = strided_cb(k, logm);
    const uint32_t tiles = uint32_t(uint64_t(1) << (logm - k - cb));
    const uint64_t n = uint64_t(1) << logm;
    const uint64_t ops = qf_intops::transform_ops(kOps, n, OP == qfd::kWht ? k : 0, OP == qfd::kMobius ? k : 0, 1, 0);
    launch(s, timed, "k_butterfly_strided", 2 * n * 16, ops, [&] {
      qfd::k_butterfly_strided<OP><<<tile_grid(tiles), qfd::kTileThreads, qfd::kTileSmem, s>>>(src, dst, logR, lo, k, cb,
                                                                                                tiles);
    });
    src = dst;
    lo += k;
  }
}

// The transform passes of one codeword (2^logm message entries in 2^(logm -
// logR) columns of R = 2^logR rows, message half at cw, parity at cw + R).
// On entry the message half holds the packed message with its Mobius levels
// [0, mob_from) applied; mob_from = logm when the message needs none (the
// extension codewords).  On return the message half holds the Mobius
// transform of the whole message (mobius_in_place, packed.rs:708-752) and
// the parity half WHT(alpha * WHT(message)) per column (qafold_short.rs:
// 975-1002).
//
// Every level is a 2 x 2 map on one index bit, and maps on different bits
// commute, so the passes group them by the bits a tile covers (12 per tile;
// the tile levels 0..11 of a column are its low 12 bits):
//   1. Mobius on the bits above the fused span (the column bits [logR, logm),
//      plus any within-column bits above 22), strided, in place;
//   2. Mobius then WHT #1 on the fused span [12, min(logR, 22)) in one
//      strided pass, writing the message (now final) and the parity;
//   3. WHT #1 on within-column bits above 22 (KoalaBear, logR = 23);
//   4. WHT #1 on bits 0..11, alpha, WHT #2 on bits 0..11: one tile pass;
//   5. WHT #2 on [12, logR), strided.
// A fused span of fewer than 6 levels leaves too few bits for the fused
// pass's register stages; its Mobius levels then join pass 1 and its WHT
// levels run as a strided pass from the message into the parity.  Columns
// shorter than one tile (logR < 12) take one tile pass per WHT.
static void encode_passes(cudaStream_t s, Fe* cw, const Fe* alpha, int logR, int logm, int mob_from, bool timed,
                          bool allow_tuning) {
  check(logm <= 30, "transform passes index a codeword of at most 2^31 elements");
  const size_t R = size_t(1) << logR;
  Fe* msg = cw;
  Fe* par = cw + R;
  const bool mobius = mob_from < logm;
  // Columns shorter than a tile (logR < 12): the rest of the Mobius
  // transform, then per WHT a tile pass (levels 0..logR, alpha first for the
  // second) and strided passes.
  if (logR < qfd::kMaxTileLog) {
    const int wl = std::min(qfd::kMaxTileLog, logR);
    if (mobius) strided_passes<qfd::kMobius>(s, msg, msg, logR, logm, mob_from, logm, timed, allow_tuning);
    for (int pass = 0; pass < 2; ++pass) {
      launch(s, timed, "k_wht_tile", (uint64_t(2) << logm) * 16,
             qf_intops::transform_ops(kOps, uint64_t(1) << logm, wl, 0, 1, pass),
             [&] { wht_tile_launch(s, pass == 0 ? msg : par, par, pass == 0 ? nullptr : alpha, logR, logm, wl); });
      strided_passes<qfd::kWht>(s, par, par, logR, logm, wl, logR, timed, allow_tuning);
    }
    return;
  }
  constexpr int kT = qfd::kMaxTileLog;
  check(!mobius || mob_from == kT, "the Mobius tile pass covers bits 0..11");
  const int top = std::min(logR, kT + 10);  // fused span [kT, top)
  const int k = top - kT;
  // KoalaBear does not fuse the Mobius and WHT #1 strided levels: its
  // butterflies reduce at every level (3 operations per element, coefficient
  // and level), so a 20-level pass is issue-bound where its separate strided
  // passes run at 0.95 of HBM (the fused plan measured 351 against 337 ms
  // per 8B step).  It still takes the WHT-alpha-WHT tile pass.
#if defined(QF_FIELD_KB)
  const bool fused = false;
#else
  const bool fused = mobius && k >= 6;
#endif
  if (mobius) strided_passes<qfd::kMobius>(s, msg, msg, logR, logm, fused ? top : kT, logm, timed, allow_tuning);
  if (fused) {
    const int cb = strided_cb(k, logm);
    const uint32_t tiles = uint32_t(uint64_t(1) << (logm - k - cb));
    launch(s, timed, "k_mobius_wht_strided", (uint64_t(3) << logm) * 16,
           qf_intops::transform_ops(kOps, uint64_t(1) << logm, k, k, 2, 0), [&] {
             qfd::k_mobius_wht_strided<<<tile_grid(tiles), qfd::kTileThreads, qfd::kTileSmem + qfd::kPrefetchSmem, s>>>(cw, uint32_t(R), logR,
                                                                                                 kT, k, cb, tiles);
           });
    strided_passes<qfd::kWht>(s, par, par, logR, logm, top, logR, timed, allow_tuning);
  } else {
    // WHT #1's levels [12, logR) as one span (the tuner's split), message
    // into parity.
    strided_passes<qfd::kWht>(s, msg, par, logR, logm, kT, logR, timed, allow_tuning);
  }
  const uint32_t tiles = uint32_t(uint64_t(1) << (logm - kT));
  const Fe* src = k > 0 ? par : msg;
  launch(s, timed, "k_wht_alpha_wht_tile", (uint64_t(2) << logm) * 16 + uint64_t(R) * 16,
         qf_intops::transform_ops(kOps, uint64_t(1) << logm, 2 * kT, 0, 2, 1), [&] {
           qfd::k_wht_alpha_wht_tile<<<tile_grid(tiles), qfd::kTileThreads, qfd::kTileSmem + qfd::kAlphaStageSmem, s>>>(
               src, par, alpha, logR, tiles);
         });
  strided_passes<qfd::kWht>(s, par, par, logR, logm, kT, logR, timed, allow_tuning);
}

// Inner levels of a row tree over the n_leaves digests at tree[0..): level j
// at digest offset level_off[j], the root last.  Launches of two levels per
// thread (k_hash_subtrees: each thread hashes a 4-child subtree, no barrier;
// three levels measured slower, their registers cost occupancy) while the
// level they reach keeps at least 2^11 nodes, then one CTA for the levels
// above (k_hash_top): 7 launches for 2^23 leaves instead of 23.
static void build_tree(cudaStream_t s, uint4* tree, uint64_t n_leaves, std::vector<uint64_t>& level_off, bool timed) {
  level_off.clear();
  for (uint64_t k = n_leaves, off = 0;; k /= 2) {
    level_off.push_back(off);
    off += k;
    if (k <= 1) break;
  }
  const ::qfd::InnerPrefix ip = inner_prefix();
  constexpr int kTopLog = 11;
  size_t j = 0;
  uint64_t n = n_leaves;
  while (n > (uint64_t(1) << kTopLog)) {
    const int L = std::min(2, ilog2(n) - kTopLog);
    qfd::TreeLevels lv{};
    for (int t = 0; t <= L; ++t) lv.off[t] = level_off[j + t];
    const uint64_t top = n >> L;
    const unsigned grid = unsigned((top + kThreads - 1) / kThreads);
    launch(s, timed, "k_hash_inner", n * 32 + (n - top) * 32, qf_intops::inner_hash_ops(n - top), [&] {
      if (L == 1) qfd::k_hash_subtrees<1><<<grid, kThreads, 0, s>>>(tree, top, lv, ip);
      else qfd::k_hash_subtrees<2><<<grid, kThreads, 0, s>>>(tree, top, lv, ip);
    });
    j += L;
    n = top;
  }
  if (n > 1) {
    qfd::TreeLevels lv{};
    for (int t = 0; t <= ilog2(n); ++t) lv.off[t] = level_off[j + t];
    launch(s, timed, "k_hash_inner", n * 32 + (n - 1) * 32, qf_intops::inner_hash_ops(n - 1),
           [&] { qfd::k_hash_top<<<1, unsigned(std::min<uint64_t>(1024, n / 2)), 0, s>>>(tree, n, lv, ip); });
  }
}

// Encode (see encode_passes), then leaf hashes and tree.
void GpuBackend::encode_and_hash(DeviceCodeword& out, const Fe* alpha, int logR, int logm, bool ext_domain, int mob_from) {
  const size_t R = size_t(1) << logR;
  encode_passes(s_, out.cw.p, alpha, logR, logm, mob_from < 0 ? logm : mob_from, true, true);
  // Leaves and inner levels.
  const uint64_t n_ext = 2 * R;
  ::qfd::LeafPrefix lp = leaf_prefix(out.n_cols, ext_domain);
  const unsigned lgrid = unsigned((n_ext + qfd::kLeafThreads - 1) / qfd::kLeafThreads);
  const uint64_t leaf_ops = qf_intops::leaf_hash_ops(n_ext, ext_domain ? 80 : 75, out.n_cols * 16);
  if (ext_domain)
    QF_LAUNCH_OPS(s_, "k_hash_leaves", n_ext * out.n_cols * 16 + n_ext * 32, leaf_ops,
                  qfd::k_hash_leaves<16><<<lgrid, qfd::kLeafThreads, 0, s_>>>(out.cw.p, n_ext, int(out.n_cols), lp, out.tree.p));
  else
    QF_LAUNCH_OPS(s_, "k_hash_leaves", n_ext * out.n_cols * 16 + n_ext * 32, leaf_ops,
                  qfd::k_hash_leaves<11><<<lgrid, qfd::kLeafThreads, 0, s_>>>(out.cw.p, n_ext, int(out.n_cols), lp, out.tree.p));
  build_tree(s_, out.tree.p, n_ext, out.level_off, true);
  uint4 r[2];
  QF_CK(cudaMemcpyAsync(r, out.tree.p + 2 * out.level_off.back(), 32, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  out.root_ = digest_from_words(r);
}

// The setup-row leaf prefix: the prefix's whole 64-byte blocks (all but a
// non-empty tail) are compressed here.
static ::qfd::SetupLeafPrefix setup_leaf_prefix(const SetupShape& shape) {
  const std::vector<uint8_t> pre = setup_row_prefix<F>(shape);
  ::qfd::SetupLeafPrefix pf;
  uint32_t h[8];
  for (int i = 0; i < 8; ++i) h[i] = kBlake2sIv[i];
  h[0] ^= 0x01010000u ^ 32u;
  const size_t blocks = (pre.size() - 1) / 64;
  for (size_t b = 0; b < blocks; ++b) blake2s_compress(h, pre.data() + 64 * b, 64 * (b + 1), false);
  for (int i = 0; i < 8; ++i) pf.mid[i] = h[i];
  pf.t0 = uint32_t(64 * blocks);
  pf.n_tail = uint32_t(pre.size() - 64 * blocks);
  uint8_t tail[64] = {0};
  std::memcpy(tail, pre.data() + 64 * blocks, pf.n_tail);
  for (int i = 0; i < 16; ++i)
    pf.tail[i] = uint32_t(tail[4 * i]) | (uint32_t(tail[4 * i + 1]) << 8) | (uint32_t(tail[4 * i + 2]) << 16) |
                 (uint32_t(tail[4 * i + 3]) << 24);
  return pf;
}

bool DeviceSetup::encode_level(const QaCode<F>& target, const QaCode<F>& current, size_t rf, const SetupShape& shape,
                               std::vector<F>& encoded, std::vector<Digest>& leaves) {
  const size_t mr = shape.message_rows, er = shape.encoded_rows, hc = shape.h_cols;
  if (shape.t_cols != 0 || er != 2 * mr || er * hc < (size_t(1) << 20) || !target.systematic_first ||
      target.index != 2 || target.message_len != mr || current.message_len != mr * rf || !is_pow2(hc) ||
      hc > current.alphas.size() * rf)
    return false;
  check(ilog2(mr * hc) <= 30, "setup level size");
  configure_tile_kernels();  // the setup may be a process's first device work
  cudaStream_t s;
  QF_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  {
    DBuf<Fe> cw(er * hc), alpha(mr);
    DBuf<uint4> lv(2 * er);
    // Column col is the message current.alphas[col / rf][(col % rf) mr ..][.. mr).
    for (size_t col = 0; col < hc; ++col)
      QF_CK(cudaMemcpyAsync(cw.p + col * er, current.alphas[col / rf].data() + (col % rf) * mr, mr * 16,
                            cudaMemcpyHostToDevice, s));
    QF_CK(cudaMemcpyAsync(alpha.p, target.alphas[1].data(), mr * 16, cudaMemcpyHostToDevice, s));
    const int logm = ilog2(mr * hc);
    encode_passes(s, cw.p, alpha.p, ilog2(mr), logm, logm, false, true);
    const ::qfd::SetupLeafPrefix pf = setup_leaf_prefix(shape);
    qfd::k_hash_setup_rows<<<unsigned((er + kThreads - 1) / kThreads), kThreads, 0, s>>>(cw.p, er, int(hc), pf, lv.p);
    QF_CK(cudaGetLastError());
    encoded.resize(er * hc);
    leaves.resize(er);
    QF_CK(cudaMemcpyAsync(encoded.data(), cw.p, er * hc * 16, cudaMemcpyDeviceToHost, s));
    QF_CK(cudaMemcpyAsync(leaves.data(), lv.p, er * 32, cudaMemcpyDeviceToHost, s));
    QF_CK(cudaStreamSynchronize(s));
  }
  QF_CK(cudaStreamDestroy(s));
  return true;
}

static std::unique_ptr<DeviceCodeword> alloc_codeword(size_t R, size_t cols, cudaStream_t s) {
  auto cw = std::make_unique<DeviceCodeword>();
  cw->stream = s;
  cw->n_ext = 2 * R;
  cw->n_cols = cols;
  cw->cw.alloc(2 * R * cols);
  cw->tree.alloc(2 * (2 * cw->n_ext));
  return cw;
}

Digest GpuBackend::encode_block(const W* bva, uint64_t active, uint64_t src_base, DeviceCodeword& cw) {
  const int logm = ilog2(P_.pcs.packed_len());
  const int logR = logm - ilog2(P_.pcs.pp->extension_columns);
  const int l0 = std::min(qfd::kMaxTileLog, logm);
  const size_t smem = qfd::kTileSmem;
  check(logm <= 30, "transform passes index a codeword of at most 2^31 elements");
  QF_LAUNCH_OPS(s_, "k_pack_mobius_tile", (uint64_t(1) << logm) * (F::kLanes * sizeof(W) + 16),
            qf_intops::transform_ops(kOps, uint64_t(1) << logm, 0, l0, 1, 0),
            qfd::k_pack_mobius_tile<<<tile_grid(uint64_t(1) << (logm - l0)), qfd::kTileThreads, smem, s_>>>(
                bva, active, src_base, cw.cw.p, logR, l0, uint32_t(uint64_t(1) << (logm - l0))));
  encode_and_hash(cw, tables_->top_alpha1(*P_.pcs.pp), logR, logm, false, l0);
  return cw.root_;
}

DeviceCodeword& GpuBackend::scratch_codeword() {
  if (!scratch_) {
    const int logm = ilog2(P_.pcs.packed_len());
    const int logR = logm - ilog2(P_.pcs.pp->extension_columns);
    scratch_ = alloc_codeword(size_t(1) << logR, P_.pcs.pp->extension_columns, s_);
  }
  return *scratch_;
}

Digest GpuBackend::commit_block(size_t b) {
  HostScope hs("commit_block");
  check(!src_, "commit_block on streamed weights");
  const int logm = ilog2(P_.pcs.packed_len());
  const int logR = logm - ilog2(P_.pcs.pp->extension_columns);
  // The implicit zero suffix repeats one codeword; reuse its root and state.
  if (b * P_.block_len >= active_ && !blocks_.empty()) {
    for (size_t k = 0; k < blocks_.size(); ++k)
      if (k * P_.block_len >= active_ && blocks_[k]) {
        if (blocks_.size() <= b) blocks_.resize(b + 1);
        roots_.resize(std::max(roots_.size(), b + 1));
        roots_[b] = roots_[k];
        return roots_[b];
      }
  }
  auto cw = alloc_codeword(size_t(1) << logR, P_.pcs.pp->extension_columns, s_);
  encode_block(bva_, active_, uint64_t(b) * P_.block_len, *cw);
  if (blocks_.size() <= b) blocks_.resize(b + 1);
  roots_.resize(std::max(roots_.size(), b + 1));
  roots_[b] = cw->root_;
  blocks_[b] = std::move(cw);
  return roots_[b];
}

std::vector<Digest> GpuBackend::commit_streamed(const BlockStream::BlockFn& per_block) {
  HostScope hs("commit_streamed");
  check(src_ != nullptr, "commit_streamed needs streamed weights");
  DeviceCodeword& cw = scratch_codeword();
  roots_.assign(P_.blocks(), Digest{});
  src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
    roots_[b] = encode_block(d, n, 0, cw);
    if (per_block) per_block(b, d, n);
  });
  if (src_->live_blocks() < P_.blocks()) {  // the zero suffix: one codeword for all
    const Digest z = encode_block(nullptr, 0, 0, cw);
    for (size_t b = src_->live_blocks(); b < P_.blocks(); ++b) roots_[b] = z;
  }
  scratch_.reset();  // back to the pool until binding needs it again
  return roots_;
}

// The same kernels as commit_block + encode_and_hash, launched without the
// per-launch timers and into caller-owned buffers.
void commit_block_into(const Parameters<F>& P, const W* d_bva, uint64_t active, size_t b, Fe* cw, uint4* tree,
                       const Fe* alpha, uint8_t* d_root, cudaStream_t s) {
  configure_tile_kernels();
  const int logm = ilog2(P.pcs.packed_len());
  const size_t cols = P.pcs.pp->extension_columns;
  const int logR = logm - ilog2(cols);
  const size_t R = size_t(1) << logR;
  check(P.pcs.pp->seq.top().message_len == R, "alpha table length");
  // Message half: pack + Mobius levels 0..11, then the rest of the encode.
  const int l0 = std::min(qfd::kMaxTileLog, logm);
  check(logm <= 30, "transform passes index a codeword of at most 2^31 elements");
  qfd::k_pack_mobius_tile<<<tile_grid(uint64_t(1) << (logm - l0)), qfd::kTileThreads, qfd::kTileSmem, s>>>(
      d_bva, active, uint64_t(b) * P.block_len, cw, logR, l0, uint32_t(uint64_t(1) << (logm - l0)));
  QF_CK(cudaGetLastError());
  encode_passes(s, cw, alpha, logR, logm, l0, false, false);
  // Row leaves, inner levels, root.
  const uint64_t n_ext = 2 * R;
  qfd::k_hash_leaves<11><<<unsigned((n_ext + qfd::kLeafThreads - 1) / qfd::kLeafThreads), qfd::kLeafThreads, 0, s>>>(
      cw, n_ext, int(cols), leaf_prefix(cols, false), tree);
  QF_CK(cudaGetLastError());
  std::vector<uint64_t> level_off;
  build_tree(s, tree, n_ext, level_off, false);
  QF_CK(cudaMemcpyAsync(d_root, tree + 2 * level_off.back(), 32, cudaMemcpyDeviceToDevice, s));
}

// The result of the last reduction kernel (finish_reduction): n elements of
// the reduction buffer's header.
std::vector<F> GpuBackend::reduce_to_host(const DBuf<Fe>& partials, uint32_t, int n) {
  check(n >= 1 && n + 1 <= qfd::kRedHeader, "reduce arity");
  std::vector<F> out(n);
  QF_CK(cudaMemcpyAsync(out.data(), partials.p + 1, n * 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  return out;
}

std::vector<F> GpuBackend::copy_to_host(const Fe* p, uint64_t n) {
  std::vector<F> out(n);
  QF_CK(cudaMemcpyAsync(out.data(), p, n * 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  return out;
}

namespace {
// The host rounds below mirror the device kernels of the same names
// (k_sum_message, k_sum_fold_message, k_eo_fold_cross, k_lb_cross,
// k_lb_fold_cross): the same field operations on canonical elements, so the
// results are the same bytes.
std::array<F, 2> sum_message_host(const std::vector<F>& v, const std::vector<F>& w) {
  const size_t h = v.size() / 2;
  F a = F::zero(), b = F::zero();
  for (size_t i = 0; i < h; ++i) {
    a += v[i] * w[i];
    b += (v[i + h] - v[i]) * (w[i + h] - w[i]);
  }
  return {a, b};
}
void sum_fold_host(std::vector<F>& v, F ch) {
  const size_t h = v.size() / 2;
  for (size_t i = 0; i < h; ++i) v[i] += ch * (v[i + h] - v[i]);
  v.resize(h);
}
std::array<F, 2> eo_cross_host(const std::vector<F>& w, const std::vector<F>& q) {
  F a = F::zero(), b = F::zero();
  for (size_t j = 0; j + 1 < w.size(); j += 2) {
    a += w[j] * q[j + 1];
    b += w[j + 1] * q[j];
  }
  return {a, b};
}
void eo_fold_host(std::vector<F>& v, F f) {
  const size_t h = v.size() / 2;
  for (size_t i = 0; i < h; ++i) v[i] = v[2 * i] + v[2 * i + 1] * f;
  v.resize(h);
}
std::array<F, 2> lb_cross_host(const std::vector<F>& L, const std::vector<F>& R) {
  const size_t h = L.size() / 2;
  F a = F::zero(), b = F::zero();
  for (size_t i = 0; i < h; ++i) {
    a += L[i] * R[h + i];
    b += L[h + i] * R[i];
  }
  return {a, b};
}
void lb_fold_host(std::vector<F>& v, F f) {
  const size_t h = v.size() / 2;
  for (size_t i = 0; i < h; ++i) v[i] += v[h + i] * f;
  v.resize(h);
}
}  // namespace

// Device table of the 2^n weights of an MSB-first point, `weights` giving the
// host table of a coordinate slice (equality_table, packed.rs:525-545, or
// tensor_weights, qafold_short_pc.rs:2826-2855; both factor over slices).
// The last <= 10 coordinates index a low table, the next <= 10 a middle
// table and the rest a high table; the high x middle product is formed on the
// device, then the full table.  Synchronises the stream before returning.
template <class W>
static void device_point_table(cudaStream_t s, const std::vector<F>& point, W weights, DBuf<Fe>& out) {
  const int n = int(point.size());
  const int lb = std::min(10, n), mb = std::min(10, n - lb), hb = n - lb - mb;
  std::vector<F> hi = weights(std::vector<F>(point.begin(), point.begin() + hb));
  std::vector<F> mid = weights(std::vector<F>(point.begin() + hb, point.begin() + hb + mb));
  std::vector<F> lo = weights(std::vector<F>(point.begin() + hb + mb, point.end()));
  DBuf<Fe> dhi(hi.size()), dmid(mid.size()), dlo(lo.size()), upper(size_t(1) << (hb + mb));
  QF_CK(cudaMemcpyAsync(dhi.p, hi.data(), hi.size() * 16, cudaMemcpyHostToDevice, s));
  QF_CK(cudaMemcpyAsync(dmid.p, mid.data(), mid.size() * 16, cudaMemcpyHostToDevice, s));
  QF_CK(cudaMemcpyAsync(dlo.p, lo.data(), lo.size() * 16, cudaMemcpyHostToDevice, s));
  const uint64_t mu = uint64_t(1) << (hb + mb), m = uint64_t(1) << n;
  QF_LAUNCH(s, "k_table", mu * 16, qfd::k_table<<<grid_for(mu, kThreads), kThreads, 0, s>>>(dhi.p, dmid.p, mb, mu, upper.p));
  if (out.n != m) out.alloc(m);
  QF_LAUNCH(s, "k_table", m * 16, qfd::k_table<<<grid_for(m, kThreads), kThreads, 0, s>>>(upper.p, dlo.p, lb, m, out.p));
  QF_CK(cudaStreamSynchronize(s));
}
static std::vector<F> eq_slice(const std::vector<F>& p) { return equality_table(p); }
static std::vector<F> tensor_slice(const std::vector<F>& p) { return tensor_weights(p); }

// Raw lane sums of blocks [b0, b0 + nb) (nb <= 8) against the equality table
// in weights_: the tensor-core kernel for F65521, else the IMAD one.
void GpuBackend::eq_project_launch(const W* bva, uint64_t active, uint64_t b0, int nb, unsigned long long* raw,
                                   unsigned grid) {
  constexpr int L = F::kLanes;
  const uint64_t m = P_.pcs.packed_len();
  const uint64_t bytes = m * 16 + m * L * sizeof(W) * uint64_t(nb);
#if !defined(QF_FIELD_KB)
  if (imma_on()) {
    QF_LAUNCH(s_, "k_eq_project_mma", bytes,
              qfd::k_eq_project_mma<<<mma_grid(), qfd::kMmaThreads, 0, s_>>>(bva, active, P_.block_len, b0, nb, m,
                                                                              weights_.p, raw));
    return;
  }
#endif
#if defined(QF_FIELD_KB)
  QF_LAUNCH(s_, "k_eq_project_blocks", bytes,
            qfd::k_eq_project_blocks<<<grid, qfd::kEqThreads, 0, s_>>>(bva, active, P_.block_len, b0, nb, m, weights_.p, raw));
#else
  QF_LAUNCH(s_, "k_eq_project_blocks", bytes,
            qfd::k_eq_project_blocks<<<grid, qfd::kEqThreads, qfd::kEqWeightSmem, s_>>>(bva, active, P_.block_len, b0, nb, m,
                                                                                     weights_.p, raw));
#endif
}

std::vector<std::vector<F>> GpuBackend::project_blocks(const std::vector<F>& outer, size_t nblocks) {
  const uint64_t m = P_.pcs.packed_len();
  if (outer.size() != size_t(ilog2(m))) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "outer point");
  device_point_table(s_, outer, eq_slice, weights_);
  constexpr int L = F::kLanes, kRaw = qfd::kEqRaw;
  static_assert(kRaw == L * qfd::kC, "raw lane sums per block");
  DBuf<unsigned long long> raw(kRaw * nblocks);
  QF_CK(cudaMemsetAsync(raw.p, 0, kRaw * nblocks * 8, s_));
  // Zero blocks (the suffix past the active entries) have vanishing lanes.
  const size_t live = std::min<size_t>(nblocks, (active_ + P_.block_len - 1) / P_.block_len);
  const unsigned grid = unsigned(std::min<uint64_t>((m + qfd::kEqChunk - 1) / qfd::kEqChunk, 148 * 4));
  if (streaming()) {  // one block per launch, as each lands in HBM
    src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
      if (b >= nblocks) return;
      eq_project_launch(d, n, 0, 1, raw.p + kRaw * b, grid);
    });
  }
  const size_t per_launch = KernelOptions::per_matrix ? 1 : size_t(qfd::kEqBlocks);
  for (size_t b0 = 0; !streaming() && b0 < live; b0 += per_launch) {
    const int nb = int(std::min<size_t>(per_launch, live - b0));
    eq_project_launch(bva_, active_, b0, nb, raw.p + kRaw * b0, grid);
  }
  std::vector<unsigned long long> h(kRaw * nblocks);
  QF_CK(cudaMemcpyAsync(h.data(), raw.p, h.size() * 8, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  // Entries are two's complement sums of exact signed totals below 2^63.
  std::vector<std::vector<F>> out(nblocks, std::vector<F>(L));
  for (size_t b = 0; b < nblocks; ++b)
    for (int j = 0; j < L; ++j)
      for (int k = 0; k < qfd::kC; ++k) {
        const int64_t v = int64_t(h[kRaw * b + qfd::kC * j + k]);
        const int64_t r = v % int64_t(F::kPrime);
        out[b][j].c[k] = typename F::Coeff(r < 0 ? r + int64_t(F::kPrime) : r);
      }
  host_v_.clear();
  host_w_.clear();
  sum_len_ = 0;
  return out;
}

const DeviceCodeword& GpuBackend::single_codeword() {
  if (!src_) return *blocks_.at(0);
  if (!single_cw_) {
    DeviceCodeword& cw = scratch_codeword();
    Digest r{};
    if (src_->live_blocks() == 0) r = encode_block(nullptr, 0, 0, cw);
    src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
      if (b == 0) r = encode_block(d, n, 0, cw);
    });
    if (r != roots_.at(0)) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
    single_cw_ = &cw;
  }
  return *single_cw_;
}

// values[i] (+)= sum_b sum_j v(b * block_len + 8i + j) T[b * L + j] over the
// packed length m: the tensor-core kernel for F65521, else the dp4a / IMAD one.
void GpuBackend::block_fold_launch(const W* bva, uint64_t active, int blocks, const Fe* T, int accumulate) {
  constexpr int L = F::kLanes;
  const uint64_t m = P_.pcs.packed_len();
  const uint64_t bytes = m * (L * sizeof(W) * uint64_t(blocks) + (accumulate ? 32 : 16));
#if !defined(QF_FIELD_KB)
  if (imma_on()) {
    QF_LAUNCH(s_, "k_block_fold_mma", bytes,
              qfd::k_block_fold_mma<<<mma_grid(), qfd::kMmaThreads, 0, s_>>>(bva, active, P_.block_len, blocks, m, T,
                                                                              values_.p, accumulate));
    return;
  }
#endif
  set_smem(qfd::k_block_fold, size_t(blocks) * L * 16);
  QF_LAUNCH(s_, "k_block_fold", bytes,
            qfd::k_block_fold<<<grid_for(m, kThreads), kThreads, size_t(blocks) * L * 16, s_>>>(
                bva, active, P_.block_len, blocks, m, T, values_.p, accumulate));
}

std::vector<F> GpuBackend::project(const std::vector<F>& outer) {
  single_cw_ = nullptr;  // a new opening
  std::vector<std::vector<F>> lanes = project_blocks(outer, 1);
  // Packed values of the single block: the block fold with weight one.
  const uint64_t m = P_.pcs.packed_len();
  values_.alloc(m);
  constexpr int L = F::kLanes;
  std::vector<F> T(L);
  for (int j = 0; j < L; ++j) T[j] = basis<F>(j);
  DBuf<Fe> dT(L);
  QF_CK(cudaMemcpyAsync(dT.p, T.data(), L * 16, cudaMemcpyHostToDevice, s_));
  if (streaming()) {
    QF_CK(cudaMemsetAsync(values_.p, 0, m * 16, s_));
    src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
      if (b == 0) block_fold_launch(d, n, 1, dT.p, 1);
    });
  } else {
    block_fold_launch(bva_, active_, 1, dT.p, 0);
  }
  host_v_.clear();
  host_w_.clear();
  sum_len_ = m;
  msg_valid_ = false;
  return lanes[0];
}

void GpuBackend::apply_images(const std::vector<F>& images) {
  check(images.size() == size_t(F::kLanes), "weight images");
  DBuf<Fe> di(F::kLanes);
  QF_CK(cudaMemcpyAsync(di.p, images.data(), F::kLanes * 16, cudaMemcpyHostToDevice, s_));
  QF_LAUNCH(s_, "k_apply_images", uint64_t(weights_.n) * 32, qfd::k_apply_images<<<grid_for(weights_.n, kThreads), kThreads, 0, s_>>>(weights_.p, weights_.n, di.p));
  QF_CK(cudaStreamSynchronize(s_));
  msg_valid_ = false;
}

Digest GpuBackend::fold_and_commit(const std::vector<F>& fw) {
  const uint64_t m = P_.pcs.packed_len();
  const int logm = ilog2(m);
  const int logR = logm - ilog2(P_.pcs.pp->extension_columns);
  const int blocks = int(fw.size());
  constexpr int L = F::kLanes;
  std::vector<F> T(size_t(blocks) * L);
  for (int b = 0; b < blocks; ++b)
    for (int j = 0; j < L; ++j) T[b * L + j] = fw[b] * basis<F>(j);
  DBuf<Fe> dT(T.size());
  QF_CK(cudaMemcpyAsync(dT.p, T.data(), T.size() * 16, cudaMemcpyHostToDevice, s_));
  values_.alloc(m);
  if (streaming()) {  // accumulate block by block; the zero blocks add nothing
    QF_CK(cudaMemsetAsync(values_.p, 0, m * 16, s_));
    src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
      if (b >= size_t(blocks)) return;
      block_fold_launch(d, n, 1, dT.p + b * L, 1);
    });
  } else if (KernelOptions::per_matrix) {  // one launch per block, accumulated
    for (int b = 0; b < blocks; ++b) {
      const uint64_t off = uint64_t(b) * P_.block_len;
      block_fold_launch(off < active_ ? bva_ + off : bva_, off < active_ ? active_ - off : 0, 1, dT.p + b * L, b > 0);
    }
  } else {
    block_fold_launch(bva_, active_, blocks, dT.p, 0);
  }
  folded_ = alloc_codeword(size_t(1) << logR, P_.pcs.pp->extension_columns, s_);
  const int l0 = std::min(qfd::kMaxTileLog, logm);
  const size_t smem = qfd::kTileSmem;
  check(logm <= 30, "transform passes index a codeword of at most 2^31 elements");
  QF_LAUNCH_OPS(s_, "k_copy_mobius_tile", (uint64_t(2) << logm) * 16,
                qf_intops::transform_ops(kOps, uint64_t(1) << logm, 0, l0, 1, 0), qfd::k_copy_mobius_tile<<<tile_grid(uint64_t(1) << (logm - l0)), qfd::kTileThreads, smem, s_>>>(
                values_.p, folded_->cw.p, logR, l0, uint32_t(uint64_t(1) << (logm - l0))));
  encode_and_hash(*folded_, tables_->top_alpha1(*P_.pcs.pp), logR, logm, false, l0);
  host_v_.clear();
  host_w_.clear();
  sum_len_ = m;
  msg_valid_ = false;
  return folded_->root_;
}

void GpuBackend::sumcheck_message(F m[2]) {
  if (!msg_valid_ && !host_v_.empty()) {
    const std::array<F, 2> r = sum_message_host(host_v_, host_w_);
    msg_[0] = r[0];
    msg_[1] = r[1];
    msg_valid_ = true;
  }
  if (!msg_valid_) {
    const int g = grid_for(sum_len_ / 2, kThreads);
    if (tc_dots(Dots::kSumMessage))
      QF_LAUNCH(s_, "k_sum_message_mma", sum_len_ * 32,
                qfd::k_sum_message_mma<<<dot_grid(sum_len_ / 2), qfd::kDotThreads, 0, s_>>>(values_.p, weights_.p, sum_len_,
                                                                                             partials_.p));
    else
      QF_LAUNCH(s_, "k_sum_message", sum_len_ * 32, qfd::k_sum_message<<<g, kThreads, 0, s_>>>(values_.p, weights_.p, sum_len_, partials_.p));
    std::vector<F> r = reduce_to_host(partials_, g, 2);
    msg_[0] = r[0];
    msg_[1] = r[1];
    msg_valid_ = true;
  }
  m[0] = msg_[0];
  m[1] = msg_[1];
}

void GpuBackend::sumcheck_fold(F ch) {
  if (host_v_.empty() && sum_len_ <= kHostTail) {
    host_v_ = copy_to_host(values_.p, sum_len_);
    host_w_ = copy_to_host(weights_.p, sum_len_);
  }
  if (!host_v_.empty()) {
    sum_fold_host(host_v_, ch);
    sum_fold_host(host_w_, ch);
    sum_len_ /= 2;
    msg_valid_ = false;
    if (sum_len_ >= 2) sumcheck_message(msg_);
    return;
  }
  if (tmp_v_.n < sum_len_ / 2) { tmp_v_.alloc(std::max<uint64_t>(sum_len_ / 2, 1)); tmp_w_.alloc(std::max<uint64_t>(sum_len_ / 2, 1)); }
  const int g = grid_for(std::max<uint64_t>(sum_len_ / 4, 1), kThreads);
  if (tc_dots(Dots::kSumFold) && sum_len_ >= 4)
    QF_LAUNCH(s_, "k_sum_fold_message_mma", sum_len_ * 48,
              qfd::k_sum_fold_message_mma<<<dot_grid(sum_len_ / 4), qfd::kDotThreads, 0, s_>>>(
                  values_.p, weights_.p, sum_len_, to_fe(ch), tmp_v_.p, tmp_w_.p, partials_.p));
  else
    QF_LAUNCH(s_, "k_sum_fold_message", sum_len_ * 48, qfd::k_sum_fold_message<<<g, kThreads, 0, s_>>>(values_.p, weights_.p, sum_len_, to_fe(ch), tmp_v_.p, tmp_w_.p, partials_.p));
  std::swap(values_, tmp_v_);
  std::swap(weights_, tmp_w_);
  sum_len_ /= 2;
  if (sum_len_ >= 2) {
    std::vector<F> r = reduce_to_host(partials_, g, 2);
    msg_[0] = r[0];
    msg_[1] = r[1];
    msg_valid_ = true;
  } else {
    msg_valid_ = false;
  }
}

F GpuBackend::sumcheck_final_value() {
  if (!host_v_.empty()) return host_v_[0];
  F v;
  QF_CK(cudaMemcpyAsync(&v, values_.p, 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  return v;
}
F GpuBackend::sumcheck_final_weight() {
  if (!host_w_.empty()) return host_w_[0];
  F v;
  QF_CK(cudaMemcpyAsync(&v, weights_.p, 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  return v;
}

// Wire records of the selected rows of codewords, gathered on the device
// into one buffer and copied back once (k_binding_records).
struct BindingRecords {
  cudaStream_t s;
  uint32_t count;
  DBuf<uint64_t> idx;
  std::vector<DBuf<uint64_t>> offsets;
  std::vector<std::pair<uint64_t, uint64_t>> segs;  // (first word, words) per codeword
  DBuf<uint64_t> buf;
  uint64_t used = 0;
  BindingRecords(cudaStream_t stream, const std::vector<size_t>& rows, uint64_t words_cap) : s(stream), count(uint32_t(rows.size())) {
    std::vector<uint64_t> id(rows.begin(), rows.end());
    idx.alloc(std::max<size_t>(id.size(), 1));
    if (!id.empty()) QF_CK(cudaMemcpyAsync(idx.p, id.data(), id.size() * 8, cudaMemcpyHostToDevice, s));
    buf.alloc(std::max<uint64_t>(words_cap, 1));
  }
  static uint64_t words(const DeviceCodeword& cw, size_t count) {
    return uint64_t(count) * (2 + 2 * uint64_t(cw.n_cols) + 4 * uint64_t(ilog2(cw.n_ext)));
  }
  // Enqueues the records of `cw`; returns its segment's index.
  size_t add(const DeviceCodeword& cw) {
    const int depth = ilog2(cw.n_ext);
    const uint64_t w = words(cw, count);
    check(used + w <= buf.n, "binding record buffer");
    offsets.emplace_back(cw.level_off.size());
    QF_CK(cudaMemcpyAsync(offsets.back().p, cw.level_off.data(), cw.level_off.size() * 8, cudaMemcpyHostToDevice, s));
    const uint64_t items = uint64_t(count) * (uint64_t(cw.n_cols) + depth + 2);
    check(items <= (uint64_t(1) << 20) * kThreads, "binding records: too many items for one launch");
    if (items)
      QF_LAUNCH(s, "k_binding_records", w * 8 + uint64_t(count) * (cw.n_cols * 16 + depth * 32),
                qfd::k_binding_records<<<grid_for(items, kThreads, 1 << 20), kThreads, 0, s>>>(
                    cw.cw.p, cw.n_ext, int(cw.n_cols), cw.tree.p, offsets.back().p, depth, idx.p, count, buf.p + used));
    segs.push_back({used, w});
    used += w;
    return segs.size() - 1;
  }
  // Copies every segment back into page-locked memory (one copy, one
  // synchronisation); the lease holds them until it is released.
  PinnedStage::Lease fetch() {
    PinnedStage::Lease l = PinnedStage::acquire(std::max<uint64_t>(used, 1) * 8);
    if (used) QF_CK(cudaMemcpyAsync(l.p, buf.p, used * 8, cudaMemcpyDeviceToHost, s));
    QF_CK(cudaStreamSynchronize(s));
    return l;
  }
};

std::vector<uint8_t> GpuBackend::binding_rows(const RowSelection& sel, const std::vector<Digest>& roots) {
  HostScope hs("binding_rows");
  ByteWriter w;
  w.bytes("QAFOLDB1", 8);
  w.len(roots.size());
  if (!sel.all && !src_) {
    // Resident blocks: every block's records and the folded codeword's in
    // one gather, then the payload in block order.
    std::vector<const DeviceCodeword*> cws;
    for (size_t b = 0; b < roots.size(); ++b) {
      const DeviceCodeword* cw = b < blocks_.size() ? blocks_[b].get() : nullptr;
      if (!cw) {  // a repeated zero block: the first committed zero block
        for (size_t k = 0; k < blocks_.size() && !cw; ++k)
          if (blocks_[k] && roots_[k] == roots[b]) cw = blocks_[k].get();
      }
      if (!cw || cw->root_ != roots[b]) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
      cws.push_back(cw);
    }
    cws.push_back(folded_.get());
    std::map<const DeviceCodeword*, size_t> seg_of;
    uint64_t cap = 0;
    for (const DeviceCodeword* cw : cws)
      if (!seg_of.count(cw)) { seg_of[cw] = 0; cap += BindingRecords::words(*cw, sel.rows.size()); }
    BindingRecords rec(s_, sel.rows, cap);
    for (auto& [cw, seg] : seg_of) seg = rec.add(*cw);
    uint64_t total = w.out.size();
    for (const DeviceCodeword* cw : cws) total += 9 + rec.segs[seg_of[cw]].second * 8;
    w.out.reserve(total);
    const PinnedStage::Lease lease = rec.fetch();
    const uint64_t* h = static_cast<const uint64_t*>(lease.p);
    for (const DeviceCodeword* cw : cws) {
      const auto [first, n] = rec.segs[seg_of[cw]];
      w.u8(0);
      w.len(sel.rows.size());
      w.bytes(h + first, n * 8);
    }
    return std::move(w.out);
  }
  auto emit_into = [&](ByteWriter& w, const DeviceCodeword& cw) {
    Rows<F> r;
    if (sel.all) {
      r.all = true;
      r.n_rows = cw.n_ext;
      r.n_cols = cw.n_cols;
      r.encoded = cw.entries();
    } else {
      auto rws = cw.rows(sel.rows);
      auto pth = cw.paths(sel.rows);
      for (size_t i = 0; i < sel.rows.size(); ++i) {
        RowQuery<F> q;
        q.row = std::move(rws[i]);
        q.path.siblings = std::move(pth[i]);
        r.partial.push_back(std::move(q));
      }
    }
    write_rows(w, r);
  };
  auto emit = [&](const DeviceCodeword& cw) { emit_into(w, cw); };
  if (src_) {
    // Recompute mode: re-encode every live block as its weights land, check
    // its root, then the zero suffix once.
    DeviceCodeword& cw = scratch_codeword();
    check(roots.size() == P_.blocks(), "block roots");
    // Passes may visit the blocks in either direction: each block's rows are
    // kept apart and appended in block order.
    std::vector<std::vector<uint8_t>> per_block(src_->live_blocks());
    src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
      if (encode_block(d, n, 0, cw) != roots[b]) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
      ByteWriter bw;
      emit_into(bw, cw);
      per_block[b] = std::move(bw.out);
    });
    for (const auto& v : per_block) w.out.insert(w.out.end(), v.begin(), v.end());
    if (src_->live_blocks() < roots.size()) {
      const Digest z = encode_block(nullptr, 0, 0, cw);
      const size_t at = w.out.size();
      emit(cw);
      const std::vector<uint8_t> zero_rows(w.out.begin() + at, w.out.end());
      for (size_t b = src_->live_blocks(); b < roots.size(); ++b) {
        if (roots[b] != z) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
        if (b > src_->live_blocks()) w.out.insert(w.out.end(), zero_rows.begin(), zero_rows.end());
      }
    }
    emit(*folded_);
    return std::move(w.out);
  }
  for (size_t b = 0; b < roots.size(); ++b) {
    const DeviceCodeword* cw = b < blocks_.size() ? blocks_[b].get() : nullptr;
    if (!cw) {  // a repeated zero block: the first committed zero block
      for (size_t k = 0; k < blocks_.size() && !cw; ++k)
        if (blocks_[k] && roots_[k] == roots[b]) cw = blocks_[k].get();
    }
    if (!cw || cw->root_ != roots[b]) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
    emit(*cw);
  }
  emit(*folded_);
  return std::move(w.out);
}

// ---------------------------------------------------------------- block shards
std::vector<F> GpuBackend::fold_values(const std::vector<F>& fw) {
  HostScope hs("fold_values");
  check(!src_, "sharded fold on streamed weights");
  const uint64_t m = P_.pcs.packed_len();
  const int blocks = int(fw.size());
  constexpr int L = F::kLanes;
  std::vector<F> T(size_t(blocks) * L);
  for (int b = 0; b < blocks; ++b)
    for (int j = 0; j < L; ++j) T[b * L + j] = fw[b] * basis<F>(j);
  DBuf<Fe> dT(T.size());
  QF_CK(cudaMemcpyAsync(dT.p, T.data(), T.size() * 16, cudaMemcpyHostToDevice, s_));
  values_.alloc(m);
  block_fold_launch(bva_, active_, blocks, dT.p, 0);
  return copy_to_host(values_.p, m);
}

Digest GpuBackend::commit_folded_values(const std::vector<F>& values) {
  HostScope hs("commit_folded_values");
  const uint64_t m = P_.pcs.packed_len();
  check(values.size() == m, "folded values length");
  const int logm = ilog2(m);
  const int logR = logm - ilog2(P_.pcs.pp->extension_columns);
  values_.alloc(m);
  QF_CK(cudaMemcpyAsync(values_.p, values.data(), m * 16, cudaMemcpyHostToDevice, s_));
  folded_ = alloc_codeword(size_t(1) << logR, P_.pcs.pp->extension_columns, s_);
  const int l0 = std::min(qfd::kMaxTileLog, logm);
  check(logm <= 30, "transform passes index a codeword of at most 2^31 elements");
  QF_LAUNCH_OPS(s_, "k_copy_mobius_tile", (uint64_t(2) << logm) * 16,
                qf_intops::transform_ops(kOps, uint64_t(1) << logm, 0, l0, 1, 0), qfd::k_copy_mobius_tile<<<tile_grid(uint64_t(1) << (logm - l0)), qfd::kTileThreads, qfd::kTileSmem, s_>>>(
                values_.p, folded_->cw.p, logR, l0, uint32_t(uint64_t(1) << (logm - l0))));
  encode_and_hash(*folded_, tables_->top_alpha1(*P_.pcs.pp), logR, logm, false, l0);
  QF_CK(cudaStreamSynchronize(s_));  // the host copy of `values` may go once this returns
  host_v_.clear();
  host_w_.clear();
  sum_len_ = m;
  msg_valid_ = false;
  return folded_->root_;
}

namespace {
// One codeword's rows in the binding payload: all rows, or the sampled rows
// with their Merkle paths (write_rows).
void write_device_rows(ByteWriter& w, const DeviceCodeword& cw, const RowSelection& sel) {
  Rows<F> r;
  if (sel.all) {
    r.all = true;
    r.n_rows = cw.n_ext;
    r.n_cols = cw.n_cols;
    r.encoded = cw.entries();
  } else {
    auto rws = cw.rows(sel.rows);
    auto pth = cw.paths(sel.rows);
    for (size_t i = 0; i < sel.rows.size(); ++i) {
      RowQuery<F> q;
      q.row = std::move(rws[i]);
      q.path.siblings = std::move(pth[i]);
      r.partial.push_back(std::move(q));
    }
  }
  write_rows(w, r);
}
}  // namespace

void GpuBackend::write_block_rows(ByteWriter& w, size_t b, const RowSelection& sel, const Digest& root) {
  check(!src_, "sharded binding on streamed weights");
  const DeviceCodeword* cw = b < blocks_.size() ? blocks_[b].get() : nullptr;
  if (!cw) {  // a repeated zero block: the first committed zero block
    for (size_t k = 0; k < blocks_.size() && !cw; ++k)
      if (blocks_[k] && roots_[k] == root) cw = blocks_[k].get();
  }
  if (!cw || cw->root_ != root) fail(QF_E_INVALID_COMMITMENT, "block root mismatch");
  write_device_rows(w, *cw, sel);
}

void GpuBackend::write_folded_rows(ByteWriter& w, const RowSelection& sel) {
  check(folded_ != nullptr, "no folded codeword");
  write_device_rows(w, *folded_, sel);
}

// ---------------------------------------------------------------- TBV / EO
std::vector<W> GpuBackend::windows(const std::vector<uint64_t>& starts, size_t stride) {
  std::vector<W> out(starts.size() * stride);
  if (starts.empty()) return out;
  if (src_ && !src_->on_device()) {  // a few entries each: read them in host memory
    for (size_t i = 0; i < starts.size(); ++i)
      for (size_t k = 0; k < stride; ++k) {
        const uint64_t g = starts[i] + k;
        out[i * stride + k] = g < active_ ? src_->host()[g] : W(0);
      }
    return out;
  }
  DBuf<uint64_t> ds(starts.size());
  DBuf<W> dout(out.size());
  QF_CK(cudaMemcpyAsync(ds.p, starts.data(), starts.size() * 8, cudaMemcpyHostToDevice, s_));
  QF_LAUNCH(s_, "k_gather_windows", uint64_t(out.size()) * 2, qfd::k_gather_windows<<<grid_for(out.size(), kThreads, 1 << 20), kThreads, 0, s_>>>(bva_, active_, ds.p, uint32_t(starts.size()),
                                                                                     int(stride), dout.p));
  QF_CK(cudaMemcpyAsync(out.data(), dout.p, out.size() * sizeof(W), cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  return out;
}

// Factor-pair tables for the TBV term kernels, built on the device in one
// launch (the host only gathers each table's factor pairs and scale).
namespace {
struct TableBuilder {
  std::vector<Fe> factors;  // two entries per factor pair
  std::vector<qfd::TableSpec> specs;
  uint32_t total = 0;
  uint32_t add(const std::array<F, 2>* f, size_t n_bits, size_t count, const F& scale) {
    qfd::TableSpec sp;
    sp.out_off = total;
    sp.count = uint32_t(count);
    sp.fac_off = uint32_t(factors.size() / 2);
    sp.n_bits = uint32_t(n_bits);
    sp.scale = to_fe(scale);
    for (size_t k = 0; k < n_bits; ++k) {
      factors.push_back(to_fe(f[k][0]));
      factors.push_back(to_fe(f[k][1]));
    }
    specs.push_back(sp);
    total += uint32_t(count);
    return sp.out_off;
  }
  // Uploads and launches; the staging buffers live in the builder until the
  // caller has synchronised the stream.
  void build(cudaStream_t s, DBuf<Fe>& out) {
    out.alloc(std::max<uint32_t>(total, 1));
    if (specs.empty()) return;
    dfac.alloc(std::max<size_t>(factors.size(), 1));
    dspec.alloc(specs.size());
    if (!factors.empty()) QF_CK(cudaMemcpyAsync(dfac.p, factors.data(), factors.size() * 16, cudaMemcpyHostToDevice, s));
    QF_CK(cudaMemcpyAsync(dspec.p, specs.data(), specs.size() * sizeof(qfd::TableSpec), cudaMemcpyHostToDevice, s));
    QF_LAUNCH(s, "k_factor_tables", uint64_t(total) * 16,
              qfd::k_factor_tables<<<grid_for(total, kThreads), kThreads, 0, s>>>(dspec.p, int(specs.size()), dfac.p, total, out.p));
  }
  DBuf<Fe> dfac;
  DBuf<qfd::TableSpec> dspec;
};

// One term's tiles: rows of 2^lb (lb <= min(12, max_lb)), high bits split
// into mid (<= 2^10) and top.  4096-row tiles amortise each tile's
// cross-thread reduction over enough products.
qfd::TermTiles term_tiles(TableBuilder& tb, const std::array<F, 2>* f, size_t nh, uint64_t offset, uint64_t rows,
                          uint32_t first_tile, const F& scale, size_t max_lb = 12) {
  qfd::TermTiles T;
  const size_t lb = std::min<size_t>(std::min<size_t>(12, max_lb), nh);
  const size_t mb = std::min<size_t>(10, nh - lb);
  const uint64_t ntiles = (rows + (uint64_t(1) << lb) - 1) >> lb;
  T.offset = offset;
  T.rows = rows;
  T.first_tile = first_tile;
  T.tile_skip = 0;
  T.lb = uint32_t(lb);
  T.mb = uint32_t(mb);
  T.lo_off = tb.add(f, lb, size_t(1) << lb, F::one());
  T.mid_off = tb.add(f + lb, mb, size_t(1) << mb, F::one());
  T.top_off = tb.add(f + lb + mb, nh - lb - mb, (ntiles + (uint64_t(1) << mb) - 1) >> mb, scale);
  return T;
}
uint64_t term_tile_count(const qfd::TermTiles& T) { return (T.rows + (uint64_t(1) << T.lb) - 1) >> T.lb; }
}  // namespace

// Lane projections (tbv.rs:288-352) of large terms: one CTA per tile of up
// to 4096 rows, tile weights from device-built factor tables.
std::vector<std::vector<std::vector<F>>> GpuBackend::project_term_groups(
    const std::vector<std::vector<const Term<F>*>>& groups, size_t stride) {
  if (streaming()) return project_groups_streamed(groups, stride);
  std::vector<std::vector<std::vector<F>>> out;
  for (const auto& g : groups) out.push_back(project_terms(g, stride));
  return out;
}

// Streamed weights: every group's tiles are cut at block boundaries (a term
// is aligned to its power-of-two length, so it lies inside one block or
// covers whole blocks, and tiles no longer than a block never straddle one);
// each block's pieces run as its weights land, and the pieces of a term are
// summed at the end.
std::vector<std::vector<std::vector<F>>> GpuBackend::project_groups_streamed(
    const std::vector<std::vector<const Term<F>*>>& groups, size_t stride) {
  HostScope hs("project_terms");
  const uint64_t bl = P_.block_len;
  const size_t live = src_->live_blocks(), G = groups.size();
  std::vector<std::vector<std::vector<F>>> out(G);
  TableBuilder tb;
  std::vector<size_t> lanes_of(G, 0);
  // pieces[b][g]: launch-local tiles of block b for group g; term_of: each piece's term
  std::vector<std::vector<std::vector<qfd::TermTiles>>> pieces(live, std::vector<std::vector<qfd::TermTiles>>(G));
  std::vector<std::vector<std::vector<size_t>>> term_of(live, std::vector<std::vector<size_t>>(G));
  std::vector<std::vector<uint64_t>> tiles_bg(live, std::vector<uint64_t>(G, 0));
  for (size_t g = 0; g < G; ++g) {
    out[g].resize(groups[g].size());
    for (size_t t = 0; t < groups[g].size(); ++t) {
      const Term<F>& term = *groups[g][t];
      const size_t low_bits = std::min<size_t>(ilog2(stride), term.factors.size());
      const size_t lanes = size_t(1) << low_bits;
      out[g][t].assign(lanes, F::zero());
      if (lanes_of[g] == 0) lanes_of[g] = lanes;
      if (lanes != lanes_of[g]) fail(QF_E_ARGUMENT, "mixed lane widths");
      check(lanes <= 64 && lanes <= bl, "at most 64 projection lanes");
      if (term.offset >= active_ || term.scale.is_zero()) continue;
      const size_t nh = term.factors.size() - low_bits;
      const uint64_t rows = std::min<uint64_t>((active_ - term.offset + lanes - 1) / lanes, term.len() / lanes);
      const qfd::TermTiles T = term_tiles(tb, term.factors.data() + low_bits, nh, term.offset, rows, 0, term.scale,
                                          size_t(ilog2(bl / lanes)));
      const uint64_t span = (uint64_t(1) << T.lb) * lanes, ntiles = term_tile_count(T);
      check(term.offset % span == 0, "projection term alignment");
      for (uint64_t i = 0; i < ntiles;) {
        const uint64_t e0 = term.offset + i * span, b = e0 / bl;
        check(b < live, "projection tile past the live blocks");
        const uint64_t i1 = std::min<uint64_t>(ntiles, i + ((b + 1) * bl - e0) / span);
        qfd::TermTiles piece = T;
        piece.offset = term.offset - b * bl;  // modulo 2^64: the kernel adds the tile's rows back
        piece.tile_skip = uint32_t(i);
        piece.first_tile = uint32_t(tiles_bg[b][g]);
        pieces[b][g].push_back(piece);
        term_of[b][g].push_back(t);
        tiles_bg[b][g] += i1 - i;
        check(tiles_bg[b][g] < (uint64_t(1) << 31), "projection tile count");
        i = i1;
      }
    }
  }
  DBuf<Fe> tables;
  tb.build(s_, tables);
  // One device array of all pieces, block-major then group; each group's tile
  // outputs block-major too, so a piece's tiles are one segment.
  std::vector<qfd::TermTiles> all;
  std::vector<std::vector<size_t>> piece_at(live, std::vector<size_t>(G));
  std::vector<std::vector<uint64_t>> tile_base(live, std::vector<uint64_t>(G));
  std::vector<uint64_t> tiles_g(G, 0);
  std::vector<std::vector<uint32_t>> seg(G, std::vector<uint32_t>(1, 0));
  std::vector<std::vector<size_t>> seg_term(G);
  for (size_t b = 0; b < live; ++b)
    for (size_t g = 0; g < G; ++g) {
      piece_at[b][g] = all.size();
      tile_base[b][g] = tiles_g[g];
      for (size_t k = 0; k < pieces[b][g].size(); ++k) {
        all.push_back(pieces[b][g][k]);
        const uint64_t end = k + 1 < pieces[b][g].size() ? pieces[b][g][k + 1].first_tile : tiles_bg[b][g];
        seg[g].push_back(uint32_t(tiles_g[g] + end));
        seg_term[g].push_back(term_of[b][g][k]);
      }
      tiles_g[g] += tiles_bg[b][g];
    }
  if (all.empty()) return out;
  DBuf<qfd::TermTiles> dall(all.size());
  QF_CK(cudaMemcpyAsync(dall.p, all.data(), all.size() * sizeof(qfd::TermTiles), cudaMemcpyHostToDevice, s_));
  std::vector<DBuf<Fe>> dtile(G);
  for (size_t g = 0; g < G; ++g) dtile[g].alloc(std::max<uint64_t>(tiles_g[g] * lanes_of[g], 1));
  src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
    for (size_t g = 0; g < G; ++g) {
      const uint64_t tiles = tiles_bg[b][g];
      if (!tiles) continue;
      project_terms_launch(d, n, dall.p + piece_at[b][g], int(pieces[b][g].size()), tiles, tables.p, lanes_of[g],
                           dtile[g].p + tile_base[b][g] * lanes_of[g], n * sizeof(W));
    }
  });
  for (size_t g = 0; g < G; ++g) {
    const size_t np = seg_term[g].size();
    if (!np) continue;
    DBuf<uint32_t> dseg(seg[g].size());
    DBuf<Fe> dpiece(np * lanes_of[g]);
    QF_CK(cudaMemcpyAsync(dseg.p, seg[g].data(), seg[g].size() * 4, cudaMemcpyHostToDevice, s_));
    QF_LAUNCH(s_, "k_sum_segments", tiles_g[g] * lanes_of[g] * 16,
              qfd::k_sum_segments<<<unsigned(np), kThreads, 0, s_>>>(dtile[g].p, dseg.p, int(lanes_of[g]), dpiece.p));
    std::vector<F> h(np * lanes_of[g]);
    QF_CK(cudaMemcpyAsync(h.data(), dpiece.p, h.size() * 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaStreamSynchronize(s_));
    for (size_t k = 0; k < np; ++k)
      for (size_t l = 0; l < lanes_of[g]; ++l) out[g][seg_term[g][k]][l] += h[k * lanes_of[g] + l];
  }
  return out;
}

// Lane projections of `n_terms` term tile lists (`tiles` tiles) into out:
// the dp4a kernel for F65521 terms of 16 lanes, the general one otherwise.
void GpuBackend::project_terms_launch(const W* bva, uint64_t active, const qfd::TermTiles* terms, int n_terms,
                                      uint64_t tiles, const Fe* tables, size_t lanes, Fe* out, uint64_t bytes) {
  const unsigned grid = unsigned((tiles + qfd::kTilesPerCta - 1) / qfd::kTilesPerCta);
#if !defined(QF_FIELD_KB)
  if (lanes == 16) {
    QF_LAUNCH(s_, "k_project_terms", bytes,
              qfd::k_project_terms16<<<grid, qfd::kTermThreads, 0, s_>>>(bva, active, terms, n_terms, uint32_t(tiles),
                                                                         tables, out));
    return;
  }
#endif
  QF_LAUNCH(s_, "k_project_terms", bytes,
            qfd::k_project_terms<<<grid, qfd::kTermThreads, 0, s_>>>(bva, active, terms, n_terms, uint32_t(tiles), tables,
                                                                     int(lanes), out));
}

std::vector<std::vector<F>> GpuBackend::project_terms(const std::vector<const Term<F>*>& terms, size_t stride) {
  if (streaming()) return project_groups_streamed({terms}, stride)[0];
  HostScope hs("project_terms");
  std::vector<std::vector<F>> out(terms.size());
  TableBuilder tb;
  std::vector<qfd::TermTiles> tt;
  std::vector<uint32_t> seg(1, 0);
  uint64_t tiles = 0, proj_bytes = 0;
  size_t common_lanes = 0;
  for (size_t t = 0; t < terms.size(); ++t) {
    const Term<F>& term = *terms[t];
    const size_t low_bits = std::min<size_t>(ilog2(stride), term.factors.size());
    const size_t lanes = size_t(1) << low_bits;
    out[t].assign(lanes, F::zero());
    if (common_lanes == 0) common_lanes = lanes;
    if (lanes != common_lanes) fail(QF_E_ARGUMENT, "mixed lane widths");
    check(lanes <= 64, "at most 64 projection lanes");
    if (term.offset < active_ && !term.scale.is_zero()) {
      const size_t nh = term.factors.size() - low_bits;
      const uint64_t rows = std::min<uint64_t>((active_ - term.offset + lanes - 1) / lanes, term.len() / lanes);
      qfd::TermTiles T = term_tiles(tb, term.factors.data() + low_bits, nh, term.offset, rows, uint32_t(tiles), term.scale);
      tiles += term_tile_count(T);
      proj_bytes += rows * lanes * sizeof(W) + term_tile_count(T) * 16;
      tt.push_back(T);
    }
    check(tiles < (uint64_t(1) << 31), "projection tile count");
    seg.push_back(uint32_t(tiles));
  }
  if (tiles == 0) return out;
  DBuf<Fe> tables, dtile(tiles * common_lanes), dterm(terms.size() * common_lanes);
  tb.build(s_, tables);
  DBuf<qfd::TermTiles> dtt(tt.size());
  DBuf<uint32_t> dseg(seg.size());
  QF_CK(cudaMemcpyAsync(dseg.p, seg.data(), seg.size() * 4, cudaMemcpyHostToDevice, s_));
  if (KernelOptions::per_matrix) {
    // One launch per term (a bucket's claim term, or a padding / suffix
    // term): each term's tiles renumbered from 0, its outputs at its first tile.
    std::vector<qfd::TermTiles> solo = tt;
    for (auto& T : solo) T.first_tile = 0;
    QF_CK(cudaMemcpyAsync(dtt.p, solo.data(), solo.size() * sizeof(qfd::TermTiles), cudaMemcpyHostToDevice, s_));
    for (size_t k = 0; k < tt.size(); ++k) {
      const uint64_t n = term_tile_count(tt[k]);
      project_terms_launch(bva_, active_, dtt.p + k, 1, n, tables.p, common_lanes,
                           dtile.p + size_t(tt[k].first_tile) * common_lanes, tt[k].rows * common_lanes * sizeof(W) + n * 16);
    }
  } else {
    QF_CK(cudaMemcpyAsync(dtt.p, tt.data(), tt.size() * sizeof(qfd::TermTiles), cudaMemcpyHostToDevice, s_));
    project_terms_launch(bva_, active_, dtt.p, int(tt.size()), tiles, tables.p, common_lanes, dtile.p, proj_bytes);
  }
  QF_LAUNCH(s_, "k_sum_segments", tiles * common_lanes * 16, qfd::k_sum_segments<<<unsigned(terms.size()), kThreads, 0, s_>>>(dtile.p, dseg.p, int(common_lanes), dterm.p));
  std::vector<F> h(terms.size() * common_lanes);
  QF_CK(cudaMemcpyAsync(h.data(), dterm.p, h.size() * 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  for (size_t t = 0; t < terms.size(); ++t)
    for (size_t l = 0; l < common_lanes; ++l) out[t][l] = h[t * common_lanes + l];
  return out;
}

void GpuBackend::cross_terms(const Query<F>& q, size_t stride, std::vector<F>& pos, std::vector<F>& neg) {
  HostScope hs("eo_cross_terms");
  pos.assign(stride - 1, F::zero());
  neg.assign(stride - 1, F::zero());
  std::vector<const Term<F>*> big, small;
  for (const auto& t : q.terms) (t.len() >= stride ? big : small).push_back(&t);
  std::vector<std::vector<F>> pr = project_terms(big, stride);
  if (!big.empty() && stride > 1) {
    std::vector<F> prs(big.size() * stride), lows(big.size() * stride);
    for (size_t i = 0; i < big.size(); ++i) {
      if (pr[i].size() != stride) fail(QF_E_ARGUMENT, "projection lanes");
      std::vector<F> low = factor_weights(big[i]->factors.data(), ilog2(stride));
      std::copy(pr[i].begin(), pr[i].end(), prs.begin() + i * stride);
      std::copy(low.begin(), low.end(), lows.begin() + i * stride);
    }
    DBuf<Fe> dpr(prs.size()), dlow(lows.size()), dout(2 * (stride - 1));
    QF_CK(cudaMemcpyAsync(dpr.p, prs.data(), prs.size() * 16, cudaMemcpyHostToDevice, s_));
    QF_CK(cudaMemcpyAsync(dlow.p, lows.data(), lows.size() * 16, cudaMemcpyHostToDevice, s_));
    QF_LAUNCH(s_, "k_laurent_cross", uint64_t(prs.size()) * 32,
              qfd::k_laurent_cross<<<unsigned(2 * (stride - 1)), kThreads, 0, s_>>>(dpr.p, dlow.p, int(big.size()), int(stride), dout.p));
    std::vector<F> h(2 * (stride - 1));
    QF_CK(cudaMemcpyAsync(h.data(), dout.p, h.size() * 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaStreamSynchronize(s_));
    for (size_t d = 1; d < stride; ++d) {
      pos[d - 1] += h[d - 1];
      neg[d - 1] += h[stride - 2 + d];
    }
  }
  std::vector<uint64_t> starts;
  for (const auto* t : small) starts.push_back(t->offset / stride * stride);
  std::vector<W> win = windows(starts, stride);
  for (size_t s = 0; s < small.size(); ++s) {
    const Term<F>& term = *small[s];
    const size_t start = starts[s];
    std::vector<F> qv(stride, F::zero());
    for (size_t i = 0; i < term.len(); ++i) qv[term.offset - start + i] = term.weight(i);
    const W* v = win.data() + s * stride;
    for (size_t d = 1; d < stride; ++d)
      for (size_t lane = 0; lane + d < stride; ++lane) {
        pos[d - 1] += qv[lane + d].mul_prime(F::small(v[lane]));
        neg[d - 1] += qv[lane].mul_prime(F::small(v[lane + d]));
      }
  }
}

// Packed EO witness rows [0, rows) of the weights at `bva` (`active`
// entries): the tensor-core kernel for F65521 at stride 16, else dp4a / IMAD.
void GpuBackend::eo_witness_launch(const W* bva, uint64_t active, uint64_t rows, size_t stride, const Fe* powers,
                                   Fe* out) {
  const uint64_t bytes = std::min<uint64_t>(active, rows * stride) * sizeof(W) + rows * 16;
#if !defined(QF_FIELD_KB)
  if (imma_on() && stride == 16) {
    QF_LAUNCH(s_, "k_eo_witness_mma", bytes,
              qfd::k_eo_witness_mma<<<mma_grid(), qfd::kMmaThreads, 0, s_>>>(bva, active, rows, powers, out));
    return;
  }
#endif
  QF_LAUNCH(s_, "k_eo_witness", bytes,
            qfd::k_eo_witness<<<grid_for(rows, kThreads), kThreads, 0, s_>>>(bva, active, rows, int(stride), powers, out));
}

F GpuBackend::eo_build(const Query<F>& q, F ch, F inv, size_t logical, size_t stride) {
  HostScope hs("eo_build");
  const uint64_t rows = logical / stride;
  eo_len_ = rows;
  host_wit_.clear();
  host_qv_.clear();
  wit_.alloc(rows);
  qv_.alloc(rows);
  std::vector<F> pinv = consecutive_powers(inv, stride);
  DBuf<Fe> dp(stride);
  QF_CK(cudaMemcpyAsync(dp.p, pinv.data(), stride * 16, cudaMemcpyHostToDevice, s_));
  if (streaming()) {
    // Rows of each block as its weights land; rows past the live blocks are zero.
    check(P_.block_len % stride == 0, "block length and EO stride");
    const uint64_t rpb = P_.block_len / stride;
    QF_CK(cudaMemsetAsync(wit_.p, 0, rows * 16, s_));
    src_->for_each(s_, [&](size_t b, const W* d, uint64_t n) {
      const uint64_t r0 = uint64_t(b) * rpb;
      if (r0 >= rows) return;
      const uint64_t rb = std::min(rpb, rows - r0);
      eo_witness_launch(d, n, rb, stride, dp.p, wit_.p + r0);
    });
  } else if (KernelOptions::per_matrix) {
    // One launch per bucket: the rows [offset / stride, end / stride) of
    // each bucket, a run of small buckets sharing a row joined to the next.
    uint64_t r0 = 0;
    for (size_t k = 0; k < P_.layout.buckets.size() && r0 < rows; ++k) {
      const auto& bk = P_.layout.buckets[k];
      const uint64_t end = k + 1 < P_.layout.buckets.size() ? (bk.offset + bk.len()) / stride : rows;
      if (end <= r0) continue;
      const uint64_t r1 = std::min(end, rows);
      const uint64_t g0 = r0 * stride;
      eo_witness_launch(bva_ + std::min<uint64_t>(g0, active_), active_ > g0 ? active_ - g0 : 0, r1 - r0, stride, dp.p,
                        wit_.p + r0);
      r0 = r1;
    }
    if (r0 < rows)
      eo_witness_launch(bva_ + std::min<uint64_t>(r0 * stride, active_), active_ > r0 * stride ? active_ - r0 * stride : 0,
                        rows - r0, stride, dp.p, wit_.p + r0);
  } else {
    eo_witness_launch(bva_, active_, rows, stride, dp.p, wit_.p);
  }
  // Query fold (tbv.rs:393-428): zero, then two disjoint passes of large-term
  // tiles, then the merged small-term contributions.
  QF_CK(cudaMemsetAsync(qv_.p, 0, rows * 16, s_));
  std::vector<F> powers = consecutive_powers(ch, stride);
  const size_t ls = ilog2(stride);
  TableBuilder tb;
  std::vector<qfd::TermTiles> pass_terms[2];
  uint64_t pass_tiles[2] = {0, 0}, query_bytes[2] = {0, 0};
  std::map<uint64_t, F> sparse;
  const size_t n_claim_terms = P_.layout.buckets.size();
  for (size_t ti = 0; ti < q.terms.size(); ++ti) {
    const Term<F>& term = q.terms[ti];
    if (term.len() >= stride) {
      std::vector<F> low = factor_weights(term.factors.data(), ls);
      F sc = F::zero();
      for (size_t j = 0; j < stride; ++j) sc += low[j] * powers[j];
      sc = term.scale * sc;
      if (sc.is_zero()) continue;
      // Claim and zero-suffix terms are disjoint; padding terms overlap claim terms.
      const int pass = (ti < n_claim_terms || term.offset >= P_.layout.active) ? 0 : 1;
      const size_t nh = term.factors.size() - ls;
      qfd::TermTiles T = term_tiles(tb, term.factors.data() + ls, nh, term.offset / stride, term.len() / stride,
                                    uint32_t(pass_tiles[pass]), sc);
      pass_tiles[pass] += term_tile_count(T);
      check(pass_tiles[pass] < (uint64_t(1) << 31), "query tile count");
      query_bytes[pass] += T.rows * 32;
      pass_terms[pass].push_back(T);
    } else {
      for (size_t i = 0; i < term.len(); ++i) {
        auto it = sparse.find(term.offset / stride);
        F add = term.weight(i) * powers[(term.offset + i) % stride];
        if (it == sparse.end()) sparse[term.offset / stride] = add; else it->second += add;
      }
    }
  }
  DBuf<Fe> tables;
  tb.build(s_, tables);
  DBuf<qfd::TermTiles> dtt[2];
  for (int pass = 0; pass < 2; ++pass) {
    auto& tl = pass_terms[pass];
    if (tl.empty()) continue;
    dtt[pass].alloc(tl.size());
    if (KernelOptions::per_matrix) {  // one launch per term, tiles renumbered from 0
      std::vector<qfd::TermTiles> solo = tl;
      for (auto& T : solo) T.first_tile = 0;
      QF_CK(cudaMemcpyAsync(dtt[pass].p, solo.data(), solo.size() * sizeof(qfd::TermTiles), cudaMemcpyHostToDevice, s_));
      for (size_t k = 0; k < tl.size(); ++k) {
        const uint64_t n = term_tile_count(tl[k]);
        QF_LAUNCH(s_, "k_query_terms", tl[k].rows * 32,
                  qfd::k_query_terms<<<unsigned((n + qfd::kTilesPerCta - 1) / qfd::kTilesPerCta), kThreads, 0, s_>>>(
                      dtt[pass].p + k, 1, uint32_t(n), tables.p, qv_.p));
      }
      continue;
    }
    QF_CK(cudaMemcpyAsync(dtt[pass].p, tl.data(), tl.size() * sizeof(qfd::TermTiles), cudaMemcpyHostToDevice, s_));
    QF_LAUNCH(s_, "k_query_terms", query_bytes[pass],
              qfd::k_query_terms<<<unsigned((pass_tiles[pass] + qfd::kTilesPerCta - 1) / qfd::kTilesPerCta), kThreads, 0, s_>>>(
                  dtt[pass].p, int(tl.size()), uint32_t(pass_tiles[pass]), tables.p, qv_.p));
  }
  if (!sparse.empty()) {
    std::vector<uint64_t> idx;
    std::vector<F> vals;
    for (auto& [k, v] : sparse) { idx.push_back(k); vals.push_back(v); }
    DBuf<uint64_t> di(idx.size());
    DBuf<Fe> dv(vals.size());
    QF_CK(cudaMemcpyAsync(di.p, idx.data(), idx.size() * 8, cudaMemcpyHostToDevice, s_));
    QF_CK(cudaMemcpyAsync(dv.p, vals.data(), vals.size() * 16, cudaMemcpyHostToDevice, s_));
    QF_LAUNCH(s_, "k_scatter_add", uint64_t(idx.size()) * 48, qfd::k_scatter_add<<<unsigned((idx.size() + kThreads - 1) / kThreads), kThreads, 0, s_>>>(di.p, dv.p, uint32_t(idx.size()), qv_.p));
    QF_CK(cudaStreamSynchronize(s_));
  }
  const int g = grid_for(std::max<uint64_t>(rows / 2, 1), kThreads);
  if (tc_dots(Dots::kEoDotCross))
    QF_LAUNCH(s_, "k_eo_dot_cross_mma", rows * 32,
              qfd::k_eo_dot_cross_mma<<<dot_grid(rows / 2), qfd::kDotThreads, 0, s_>>>(wit_.p, qv_.p, rows, partials_.p));
  else
    QF_LAUNCH(s_, "k_eo_dot_cross", rows * 32, qfd::k_eo_dot_cross<<<g, kThreads, 0, s_>>>(wit_.p, qv_.p, rows, partials_.p));
  std::vector<F> r = reduce_to_host(partials_, g, 3);
  cross_ = {r[1], r[2]};
  if (rows == 1) {  // a single packed row has no binary rounds
    F w0, q0;
    QF_CK(cudaMemcpyAsync(&w0, wit_.p, 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaMemcpyAsync(&q0, qv_.p, 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaStreamSynchronize(s_));
    return w0 * q0;
  }
  return r[0];
}

void GpuBackend::eo_round_fold(F inv, F ch) {
  HostScope hs("eo_round_fold");
  const uint64_t n = eo_len_;
  if (host_wit_.empty() && n <= kHostTail) {
    host_wit_ = copy_to_host(wit_.p, n);
    host_qv_ = copy_to_host(qv_.p, n);
  }
  if (!host_wit_.empty()) {
    eo_fold_host(host_wit_, inv);
    eo_fold_host(host_qv_, ch);
    eo_len_ = n / 2;
    if (eo_len_ >= 2) cross_ = eo_cross_host(host_wit_, host_qv_);
    return;
  }
  const int g = grid_for(std::max<uint64_t>(n / 4, 1), kThreads);
  if (n >= (uint64_t(1) << 26)) {
    // Large rounds fold the two vectors one after the other through one
    // spare buffer (wit2_, n/2 entries at the first large round): the
    // witness folds into the spare, its old buffer becomes the spare and
    // takes the folded query, and the query's old buffer becomes the spare.
    // The rounds hold 2.5 vector lengths and allocate nothing after the
    // first (a nearly full HBM would otherwise evict and re-allocate).
    if (wit2_.n < n / 2) wit2_.alloc(n / 2);
    QF_LAUNCH(s_, "k_eo_fold_vec", n * 24, qfd::k_eo_fold_vec<<<grid_for(n / 2, kThreads), kThreads, 0, s_>>>(wit_.p, n, to_fe(inv), wit2_.p));
    std::swap(wit_, wit2_);
    if (tc_dots(Dots::kEoFoldQueryCross))
      QF_LAUNCH(s_, "k_eo_fold_query_cross_mma", n * 32,
                qfd::k_eo_fold_query_cross_mma<<<dot_grid(n / 4), qfd::kDotThreads, 0, s_>>>(wit_.p, qv_.p, n, to_fe(ch),
                                                                                             wit2_.p, partials_.p));
    else
      QF_LAUNCH(s_, "k_eo_fold_query_cross", n * 32, qfd::k_eo_fold_query_cross<<<g, kThreads, 0, s_>>>(wit_.p, qv_.p, n, to_fe(ch), wit2_.p, partials_.p));
    std::swap(qv_, wit2_);
  } else {
    if (wit2_.n < n / 2) wit2_.alloc(n / 2);
    if (qv2_.n < n / 2) qv2_.alloc(n / 2);
    if (tc_dots(Dots::kEoFoldCross) && n >= 4)
      QF_LAUNCH(s_, "k_eo_fold_cross_mma", n * 48,
                qfd::k_eo_fold_cross_mma<<<dot_grid(n / 4), qfd::kDotThreads, 0, s_>>>(wit_.p, qv_.p, n, to_fe(inv),
                                                                                       to_fe(ch), wit2_.p, qv2_.p,
                                                                                       partials_.p));
    else
      QF_LAUNCH(s_, "k_eo_fold_cross", n * 48, qfd::k_eo_fold_cross<<<g, kThreads, 0, s_>>>(wit_.p, qv_.p, n, to_fe(inv), to_fe(ch), wit2_.p, qv2_.p, partials_.p));
    std::swap(wit_, wit2_);
    std::swap(qv_, qv2_);
  }
  eo_len_ = n / 2;
  if (eo_len_ >= 2) {
    std::vector<F> r = reduce_to_host(partials_, g, 2);
    cross_ = {r[0], r[1]};
  }
}

std::array<F, 2> GpuBackend::eo_terminal() {
  F w0, q0;
  if (!host_wit_.empty()) {
    w0 = host_wit_[0];
    q0 = host_qv_[0];
    host_wit_.clear();
    host_qv_.clear();
  } else {
    QF_CK(cudaMemcpyAsync(&w0, wit_.p, 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaMemcpyAsync(&q0, qv_.p, 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaStreamSynchronize(s_));
  }
  // The EO vectors (up to 2 x 1.5 x N/stride elements) are done: give their
  // memory back before the batch opening allocates its own.
  wit_.reset();
  qv_.reset();
  wit2_.reset();
  qv2_.reset();
  return {w0, q0};
}


// ---------------------------------------------------------------- top round / Decide on device
const Fe* GpuBackend::level_alpha(size_t level, int which) { return tables_->alpha(*P_.pcs.pp, level, which); }

// MSB-first monomial tensor weights (tensor_weights, qafold_short_pc.rs:2826-2855):
// the last <= 10 coordinates index a low table, the rest a high table.
void GpuBackend::tensor_table(const std::vector<F>& point, DBuf<Fe>& out) { device_point_table(s_, point, tensor_slice, out); }

// Unnormalised WHT of a device vector of 2^logn entries, optionally
// multiplying by alpha first (one tile pass, then strided passes).
void GpuBackend::wht_dev(Fe* v, int logn, const Fe* alpha) {
  const int wl = std::min(qfd::kMaxTileLog, logn);
  QF_LAUNCH(s_, "k_wht_tile", (uint64_t(2) << logn) * 16, wht_tile_launch(s_, v, v, alpha, logn, logn, wl));
  strided_passes<qfd::kWht>(s_, v, v, logn, logn, wl, logn);
}

F GpuBackend::dot_dev(const Fe* a, const Fe* b, uint64_t n) {
  if (tc_dots(Dots::kDot)) {
    QF_LAUNCH(s_, "k_dot_mma", n * 32, qfd::k_dot_mma<<<dot_grid(n), qfd::kDotThreads, 0, s_>>>(a, b, n, partials_.p));
    return reduce_to_host(partials_, 0, 1)[0];
  }
  const int g = grid_for(n, kThreads);
  QF_LAUNCH(s_, "k_dot", n * 32, qfd::k_dot<<<g, kThreads, 0, s_>>>(a, b, n, partials_.p));
  return reduce_to_host(partials_, g, 1)[0];
}

std::array<F, 2> GpuBackend::lb_cross(const Fe* L, const Fe* R, uint64_t n) {
  const int g = grid_for(std::max<uint64_t>(n / 2, 1), kThreads);
  if (tc_dots(Dots::kLbCross))
    QF_LAUNCH(s_, "k_lb_cross_mma", n * 32, qfd::k_lb_cross_mma<<<dot_grid(n / 2), qfd::kDotThreads, 0, s_>>>(L, R, n, partials_.p));
  else
    QF_LAUNCH(s_, "k_lb_cross", n * 32, qfd::k_lb_cross<<<g, kThreads, 0, s_>>>(L, R, n, partials_.p));
  std::vector<F> r = reduce_to_host(partials_, g, 2);
  return {r[0], r[1]};
}

// prove_litebullet (qafold_short_pc.rs:1895-1940) on device vectors; with
// check_and_absorb = false it is the MultiEval row phase (no claim check, no
// domain label) and `claimed` is the running right-hand side.
LiteBullet<F> GpuBackend::litebullet_dev(F claimed, Fe* L, Fe* R, uint64_t n, PcsTranscript<F>& t, const char* label,
                                         const char* fold_label, bool check_and_absorb) {
  // Vectors of at most kHostTail elements fold on the host from the start;
  // longer ones switch there once they have folded down to that length.
  std::vector<F> hl, hr;
  if (n > 0 && n <= kHostTail) {
    hl = copy_to_host(L, n);
    hr = copy_to_host(R, n);
  }
  if (check_and_absorb) {
    if (n == 0 || !is_pow2(n)) fail(QF_E_INVALID_COMMITMENT, "litebullet claim");
    F dot = F::zero();
    if (hl.empty()) dot = dot_dev(L, R, n);
    else
      for (uint64_t i = 0; i < n; ++i) dot += hl[i] * hr[i];
    if (dot != claimed) fail(QF_E_INVALID_COMMITMENT, "litebullet claim");
    t.absorb_str("litebullet-domain", label);
  }
  F rhs = claimed;
  LiteBullet<F> out;
  std::array<F, 2> cr{F::zero(), F::zero()};
  if (n > 1) cr = hl.empty() ? lb_cross(L, R, n) : lb_cross_host(hl, hr);
  while (n > 1) {
    t.push_response(cr[0]);
    t.push_response(cr[1]);
    F ch = t.challenge_nonzero(fold_label);
    F inv = ch.inverse();
    rhs += cr[0] * ch + cr[1] * inv;
    out.a_point.push_back(inv);
    out.b_point.push_back(ch);
    if (hl.empty() && n <= kHostTail) {
      hl = copy_to_host(L, n);
      hr = copy_to_host(R, n);
    }
    if (!hl.empty()) {
      lb_fold_host(hl, inv);
      lb_fold_host(hr, ch);
      n /= 2;
      if (n > 1) cr = lb_cross_host(hl, hr);
      continue;
    }
    const int g = grid_for(std::max<uint64_t>(n / 4, 1), kThreads);
    if (tc_dots(Dots::kLbFold) && n >= 4)
      QF_LAUNCH(s_, "k_lb_fold_cross_mma", n * 48,
                qfd::k_lb_fold_cross_mma<<<dot_grid(n / 4), qfd::kDotThreads, 0, s_>>>(L, R, n, to_fe(inv), to_fe(ch),
                                                                                       partials_.p));
    else
      QF_LAUNCH(s_, "k_lb_fold_cross", n * 48,
                qfd::k_lb_fold_cross<<<g, kThreads, 0, s_>>>(L, R, n, to_fe(inv), to_fe(ch), partials_.p));
    n /= 2;
    if (n > 1) {
      std::vector<F> r = reduce_to_host(partials_, g, 2);
      cr = {r[0], r[1]};
    }
  }
  if (!hl.empty()) {
    out.a_value = hl[0];
    out.b_value = hr[0];
  } else {
    QF_CK(cudaMemcpyAsync(&out.a_value, L, 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaMemcpyAsync(&out.b_value, R, 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaStreamSynchronize(s_));
  }
  t.push_response(out.a_value);
  t.push_response(out.b_value);
  if (check_and_absorb && out.a_value * out.b_value != rhs) fail(QF_E_INVALID_COMMITMENT, "litebullet terminal");
  lb_rhs_ = rhs;
  return out;
}

// Row projection of the systematic half at tensor_weights(point[col_log..]),
// keeping the row weights in HBM for the top round.
std::vector<F> GpuBackend::open_top(const DeviceCodeword& cw, const std::vector<F>& point, size_t col_log) {
  HostScope hs("open_top");
  open_cw_ = &cw;
  const uint64_t n_rows = cw.n_ext / 2;
  tensor_table(std::vector<F>(point.begin() + col_log, point.end()), rw_d_);
  if (rw_d_.n != n_rows) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "top row weights");
  F one = F::one();
  DBuf<Fe> hi(1);
  QF_CK(cudaMemcpyAsync(hi.p, &one, 16, cudaMemcpyHostToDevice, s_));
  const int chunks = int(std::min<uint64_t>(64, (n_rows + kThreads - 1) / kThreads));
  DBuf<Fe> part(cw.n_cols * chunks);
  dim3 grid(chunks, unsigned(cw.n_cols));
  QF_LAUNCH(s_, "k_row_project", n_rows * cw.n_cols * 16 + n_rows * 16,
            qfd::k_row_project<<<grid, kThreads, 0, s_>>>(cw.cw.p, cw.n_ext, n_rows, hi.p, rw_d_.p, ilog2(n_rows), part.p));
  std::vector<F> hp(cw.n_cols * chunks);
  QF_CK(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  std::vector<F> out(cw.n_cols, F::zero());
  for (size_t c = 0; c < cw.n_cols; ++c)
    for (int k = 0; k < chunks; ++k) out[c] += hp[c * chunks + k];
  return out;
}

// prove_base_round_with_next_layer + prove_round_reductions
// (qafold_short_pc.rs:1120-1280, 1454-1527) with the vectors in HBM.
RoundOutput<F> GpuBackend::prove_top_round(const PcsParams<F>& pp, size_t level, const std::vector<F>& point,
                                           const std::vector<F>& opening, PcsTranscript<F>& t) {
  HostScope hs("opening_round");
  if (!open_cw_) fail(QF_E_ENCODING, "top round without an opened codeword");
  const DeviceCodeword& cw = *open_cw_;
  const QaCode<F>& code = pp.seq.codes[level];
  const QaCode<F>* next = level > 0 ? &pp.seq.codes[level - 1] : nullptr;
  const uint64_t n_rows = code.message_len, n_ext = cw.n_ext;
  const size_t n_cols = cw.n_cols, col_log = ilog2(n_cols);
  const int logR = ilog2(n_rows);
  if (n_ext != 2 * n_rows || rw_d_.n != n_rows || point.size() != col_log + size_t(logR))
    fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "top round dims");
  t.absorb_digest("round-root", cw.root());
  for (const F& o : opening) t.push_response(o);
  std::vector<F> freivalds;
  for (size_t i = 0; i < n_cols; ++i) freivalds.push_back(t.challenge_ext("freivalds"));
  F fv = inner_product(opening, freivalds);
  DBuf<Fe> folded(n_rows), dfw(n_cols);
  QF_CK(cudaMemcpyAsync(dfw.p, freivalds.data(), n_cols * 16, cudaMemcpyHostToDevice, s_));
  QF_LAUNCH(s_, "k_row_fold", n_rows * n_cols * 16 + n_rows * 16,
            qfd::k_row_fold<<<grid_for(n_rows, kThreads), kThreads, 0, s_>>>(cw.cw.p, n_ext, n_rows, int(n_cols), dfw.p, folded.p));
  RoundOutput<F> out;
  if (next) {
    // The folded vector is the next level's column-major message.
    const uint64_t rn = next->message_len;
    auto ncw = alloc_codeword(rn, n_cols, s_);
    QF_LAUNCH(s_, "k_to_message_halves", n_rows * 32,
              qfd::k_to_message_halves<<<grid_for(n_rows, kThreads), kThreads, 0, s_>>>(folded.p, n_rows, ilog2(rn), ncw->cw.p));
    encode_and_hash(*ncw, level_alpha(level - 1, 1), ilog2(rn), logR, true);
    absorb_next_layer(t, true, ncw->root());
    out.next_cw = std::move(ncw);
  } else {
    std::vector<F> term(n_rows);
    QF_CK(cudaMemcpyAsync(term.data(), folded.p, n_rows * 16, cudaMemcpyDeviceToHost, s_));
    QF_CK(cudaStreamSynchronize(s_));
    absorb_next_layer(t, false, hash_terminal_vector(term));
    out.terminal = std::move(term);
  }
  size_t qc = pp.num_queries(level, n_ext);
  Digest seed = t.challenge_digest("row-selection");
  RowSelection sel = make_selection(qc, n_ext, seed);
  std::vector<F> sampled(sel.size());
  std::vector<uint64_t> sel_rows;
  if (sel.all) {
    std::vector<F> all = cw.entries();
    for (uint64_t r = 0; r < n_ext; ++r) {
      F s = F::zero();
      for (size_t c = 0; c < n_cols; ++c) s += freivalds[c] * all[c * n_ext + r];
      sampled[r] = s;
      sel_rows.push_back(r);
    }
    out.rows.all = true;
    out.rows.n_rows = n_ext;
    out.rows.n_cols = n_cols;
    out.rows.encoded = std::move(all);
  } else {
    auto rws = cw.rows(sel.rows);
    auto pth = cw.paths(sel.rows);
    for (size_t i = 0; i < sel.size(); ++i) {
      RowQuery<F> q;
      q.row = std::move(rws[i]);
      q.path.siblings = std::move(pth[i]);
      F s = F::zero();
      for (size_t c = 0; c < n_cols; ++c) s += freivalds[c] * q.row[c];
      sampled[i] = s;
      out.rows.partial.push_back(std::move(q));
      sel_rows.push_back(sel.rows[i]);
    }
  }
  t.absorb_exts("sampled-values", sampled);
  // ---- round reductions
  size_t sel_log = ilog2(next_pow2(sel.size()));
  std::vector<F> sel_point;
  for (size_t i = 0; i < sel_log; ++i) sel_point.push_back(t.challenge_ext("selection-left"));
  std::vector<F> sw = tensor_weights_prefix(sel_point, sel.size());
  F selected = inner_product(sw, sampled);
  DBuf<Fe> pi(n_ext), comb(n_rows), gen_right(n_ext), tw;
  {
    DBuf<uint64_t> didx(sel_rows.size());
    DBuf<Fe> dval(sw.size());
    QF_CK(cudaMemsetAsync(pi.p, 0, n_ext * 16, s_));
    QF_CK(cudaMemcpyAsync(didx.p, sel_rows.data(), sel_rows.size() * 8, cudaMemcpyHostToDevice, s_));
    QF_CK(cudaMemcpyAsync(dval.p, sw.data(), sw.size() * 16, cudaMemcpyHostToDevice, s_));
    QF_LAUNCH(s_, "k_scatter_set", uint64_t(sw.size()) * 24,
              qfd::k_scatter_set<<<unsigned((sw.size() + kThreads - 1) / kThreads), kThreads, 0, s_>>>(pi.p, didx.p, dval.p,
                                                                                                  uint32_t(sw.size())));
    QF_CK(cudaStreamSynchronize(s_));
  }
  // generator_left_projection: WHT(alpha1 * WHT(pi[R..2R))) + pi[0..R)
  QF_CK(cudaMemcpyAsync(comb.p, pi.p + n_rows, n_rows * 16, cudaMemcpyDeviceToDevice, s_));
  wht_dev(comb.p, logR, nullptr);
  wht_dev(comb.p, logR, level_alpha(level, 1));
  QF_LAUNCH(s_, "k_add", n_rows * 48, qfd::k_add<<<grid_for(n_rows, kThreads), kThreads, 0, s_>>>(comb.p, pi.p, n_rows));
  F rho = t.challenge_ext("opening-batch");
  F combined_value = selected + rho * fv;
  QF_LAUNCH(s_, "k_axpy", n_rows * 48, qfd::k_axpy<<<grid_for(n_rows, kThreads), kThreads, 0, s_>>>(comb.p, rw_d_.p, n_rows, to_fe(rho)));
  LiteBullet<F> msg = litebullet_dev(combined_value, comb.p, folded.p, n_rows, t, "message-litebullet", "litebullet-fold", true);
  std::vector<F> pt_rows(point.begin() + col_log, point.end());
  F ole = tensor_inner_product(pt_rows, msg.a_point);
  F sle = msg.a_value - rho * ole;
  // generator_right_projection = encode(tensor_weights(a_point))
  tensor_table(msg.a_point, tw);
  QF_CK(cudaMemcpyAsync(gen_right.p, tw.p, n_rows * 16, cudaMemcpyDeviceToDevice, s_));
  QF_CK(cudaMemcpyAsync(gen_right.p + n_rows, tw.p, n_rows * 16, cudaMemcpyDeviceToDevice, s_));
  wht_dev(gen_right.p + n_rows, logR, nullptr);
  wht_dev(gen_right.p + n_rows, logR, level_alpha(level, 1));
  LiteBullet<F> gen = litebullet_dev(sle, pi.p, gen_right.p, n_ext, t, "generator-litebullet", "litebullet-fold", true);
  out.reduction = {msg.b_value, msg.b_point, gen.b_value, gen.b_point, msg.a_point};
  open_cw_ = nullptr;
  return out;
}

// MultiEval over one level's alpha columns (qafold_short_decide.rs:466-536)
// with the row vectors in HBM, followed by the direct-interleaved block fold.
bool GpuBackend::multi_eval(const PcsParams<F>& pp, size_t level, const std::vector<EvalClaim<F>>& claims,
                            const std::vector<F>* carry_message, size_t log_rows, size_t log_cols, size_t row_factor,
                            PcsTranscript<F>& t, MultiEvalOut<F>& out) {
  const QaCode<F>& code = pp.seq.codes[level];
  const uint64_t rows = uint64_t(1) << log_rows;
  if (rows < 1024 || code.alphas.size() > 2) return false;
  HostScope hs("decide_multi_eval");
  const size_t real = code.alphas.size() + (carry_message ? 1 : 0);
  if (rows != code.message_len) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "multi-eval rows");
  validate_multi_eval(claims, real, log_rows, log_cols);
  absorb_multi_eval_statement(claims, log_rows, log_cols, t);
  F rho = t.challenge_ext("multi-eval-batch");
  std::vector<DBuf<Fe>> row_w(claims.size());
  for (size_t i = 0; i < claims.size(); ++i) tensor_table(claims[i].row_point, row_w[i]);
  std::vector<const Fe*> col(real);
  for (size_t sidx = 0; sidx < code.alphas.size(); ++sidx) col[sidx] = level_alpha(level, int(sidx));
  DBuf<Fe> carry_d;
  if (carry_message) {
    // Entries past the carried message's length count as zero.
    if (carry_message->size() > rows) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "carry message length");
    carry_d.alloc(rows);
    QF_CK(cudaMemsetAsync(carry_d.p, 0, rows * 16, s_));
    QF_CK(cudaMemcpyAsync(carry_d.p, carry_message->data(), carry_message->size() * 16, cudaMemcpyHostToDevice, s_));
    col[real - 1] = carry_d.p;
  }
  std::vector<std::vector<F>> se(claims.size(), std::vector<F>(real));
  for (size_t i = 0; i < claims.size(); ++i)
    for (size_t sidx = 0; sidx < real; ++sidx) se[i][sidx] = dot_dev(row_w[i].p, col[sidx], rows);
  MultiEvalColumns<F> mc = multi_eval_columns(claims, real, log_cols, rho, se, t);
  DBuf<Fe> right(rows), folded(rows), left(rows);
  QF_CK(cudaMemsetAsync(right.p, 0, rows * 16, s_));
  QF_CK(cudaMemsetAsync(folded.p, 0, rows * 16, s_));
  for (size_t i = 0; i < claims.size(); ++i)
    QF_LAUNCH(s_, "k_axpy", rows * 48,
              qfd::k_axpy<<<grid_for(rows, kThreads), kThreads, 0, s_>>>(right.p, row_w[i].p, rows, to_fe(mc.row_scale[i])));
  for (const auto& [src, coef] : mc.terms0)
    QF_LAUNCH(s_, "k_axpy", rows * 48,
              qfd::k_axpy<<<grid_for(rows, kThreads), kThreads, 0, s_>>>(folded.p, col[src], rows, to_fe(coef)));
  QF_CK(cudaMemcpyAsync(left.p, folded.p, rows * 16, cudaMemcpyDeviceToDevice, s_));
  LiteBullet<F> lb = litebullet_dev(mc.rhs, left.p, right.p, rows, t, nullptr, "multi-eval-fold", false);
  std::vector<F> a_point = mc.a_point, b_point = mc.b_point;
  a_point.insert(a_point.end(), lb.a_point.begin(), lb.a_point.end());
  b_point.insert(b_point.end(), lb.b_point.begin(), lb.b_point.end());
  F ew = expected_weight_eval(claims, mc.powers, log_cols, b_point);
  out = MultiEvalOut<F>();
  out.ok = (lb.a_value * lb.b_value == lb_rhs_) && (lb.b_value == ew);
  out.reduced = {lb.a_value, a_point};
  // Block fold at the first log2(row_factor) coordinates of the merged row point.
  const int block_log = ilog2(row_factor);
  if (a_point.size() < log_cols + size_t(block_log)) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "merged point");
  std::vector<F> bw = tensor_weights(std::vector<F>(a_point.begin() + log_cols, a_point.begin() + log_cols + block_log));
  const uint64_t trows = rows / row_factor;
  DBuf<Fe> dbw(row_factor), rec(trows);
  QF_CK(cudaMemcpyAsync(dbw.p, bw.data(), row_factor * 16, cudaMemcpyHostToDevice, s_));
  QF_LAUNCH(s_, "k_block_combine", rows * 16 + trows * 16,
            qfd::k_block_combine<<<grid_for(trows, kThreads), kThreads, 0, s_>>>(folded.p, trows, int(row_factor), dbw.p, rec.p));
  out.folded_vector.resize(trows);
  QF_CK(cudaMemcpyAsync(out.folded_vector.data(), rec.p, trows * 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  return true;
}

// The carry's commit_extension_matrix (qafold_short_pc.rs:2327-2362) on the
// device: the column-major message becomes the codeword's message halves,
// then the same encode and extension-row hashing as a top round's next layer.
std::unique_ptr<CodewordView<F>> GpuBackend::commit_carry(const PcsParams<F>& pp, size_t code_index,
                                                          const std::vector<F>& message, size_t n_cols) {
  const QaCode<F>& code = pp.seq.codes[code_index];
  const uint64_t R = code.message_len, total = uint64_t(R) * n_cols;
  if (R < 128 || message.size() != total || !is_pow2(n_cols)) return nullptr;
  HostScope hs("decide_carry_commit_dev");
  DBuf<Fe> msg(total);
  QF_CK(cudaMemcpyAsync(msg.p, message.data(), total * 16, cudaMemcpyHostToDevice, s_));
  auto ncw = alloc_codeword(R, n_cols, s_);
  QF_LAUNCH(s_, "k_to_message_halves", total * 32,
            qfd::k_to_message_halves<<<grid_for(total, kThreads), kThreads, 0, s_>>>(msg.p, total, ilog2(R), ncw->cw.p));
  encode_and_hash(*ncw, tables_->alpha(pp, code_index, 1), ilog2(R), ilog2(total), true);
  return ncw;
}

// prove_short_qa_direct_code_switch_carry (qafold_short_decide_carry.rs:940-1027)
// with the message-length vectors in HBM.
bool GpuBackend::direct_switch(const QaCode<F>& target, size_t target_level, size_t row_factor, const RowSelection& sel,
                               const std::vector<F>& iota, const std::vector<F>& folded_message, F merged_value,
                               const std::vector<F>& merged_left, PcsTranscript<F>& t, SwitchCarry<F>& out) {
  HostScope hs("decide_switch");
  const uint64_t n = target.message_len, n_enc = target.codeword_len();
  if (n < 1024) return false;
  const int logn = ilog2(n);
  const size_t block_log = ilog2(row_factor);
  std::vector<F> base_point(merged_left.begin() + block_log, merged_left.end());
  if (folded_message.size() != n || base_point.size() != size_t(logn)) fail(QF_E_INVALID_NUMBER_OF_VARIABLES, "switch message");
  // The merged value is the message's MLE at the base point: <message, tensor weights>.
  DBuf<Fe> sparse(n_enc), comb(n), msg_d(n), ml, gr(n_enc), tw;
  QF_CK(cudaMemcpyAsync(msg_d.p, folded_message.data(), n * 16, cudaMemcpyHostToDevice, s_));
  tensor_table(base_point, ml);
  if (dot_dev(msg_d.p, ml.p, n) != merged_value) fail(QF_E_INVALID_COMMITMENT, "switch merged value");
  absorb_direct_switch(t, target, target_level, row_factor, sel, iota, merged_value, merged_left);
  size_t sel_log = ilog2(next_pow2(sel.size()));
  std::vector<F> slp;
  for (size_t i = 0; i < sel_log; ++i) slp.push_back(t.challenge_ext("direct-code-switch-selection-left"));
  std::vector<F> sl = tensor_weights_prefix(slp, sel.size());
  F selected = inner_product(sl, iota);
  std::vector<uint64_t> rows_idx;
  for (size_t i = 0; i < sel.size(); ++i) rows_idx.push_back(sel.at(i));
  {
    DBuf<uint64_t> didx(rows_idx.size());
    DBuf<Fe> dval(sl.size());
    QF_CK(cudaMemsetAsync(sparse.p, 0, n_enc * 16, s_));
    QF_CK(cudaMemcpyAsync(didx.p, rows_idx.data(), rows_idx.size() * 8, cudaMemcpyHostToDevice, s_));
    QF_CK(cudaMemcpyAsync(dval.p, sl.data(), sl.size() * 16, cudaMemcpyHostToDevice, s_));
    QF_LAUNCH(s_, "k_scatter_set", uint64_t(sl.size()) * 24,
              qfd::k_scatter_set<<<unsigned((sl.size() + kThreads - 1) / kThreads), kThreads, 0, s_>>>(sparse.p, didx.p, dval.p,
                                                                                                  uint32_t(sl.size())));
    QF_CK(cudaStreamSynchronize(s_));
  }
  const Fe* alpha = level_alpha(target_level, 1);
  QF_CK(cudaMemcpyAsync(comb.p, sparse.p + n, n * 16, cudaMemcpyDeviceToDevice, s_));
  wht_dev(comb.p, logn, nullptr);
  wht_dev(comb.p, logn, alpha);
  QF_LAUNCH(s_, "k_add", n * 48, qfd::k_add<<<grid_for(n, kThreads), kThreads, 0, s_>>>(comb.p, sparse.p, n));
  F rho = t.challenge_ext("direct-code-switch-opening-batch");
  F combined = selected + rho * merged_value;
  QF_LAUNCH(s_, "k_axpy", n * 48, qfd::k_axpy<<<grid_for(n, kThreads), kThreads, 0, s_>>>(comb.p, ml.p, n, to_fe(rho)));
  LiteBullet<F> msg = litebullet_dev(combined, comb.p, msg_d.p, n, t, "decide-direct-carry-message-litebullet", "litebullet-fold", true);
  F ole = tensor_inner_product(base_point, msg.a_point);
  F sle = msg.a_value - rho * ole;
  tensor_table(msg.a_point, tw);
  QF_CK(cudaMemcpyAsync(gr.p, tw.p, n * 16, cudaMemcpyDeviceToDevice, s_));
  QF_CK(cudaMemcpyAsync(gr.p + n, tw.p, n * 16, cudaMemcpyDeviceToDevice, s_));
  wht_dev(gr.p + n, logn, nullptr);
  wht_dev(gr.p + n, logn, alpha);
  LiteBullet<F> gen = litebullet_dev(sle, sparse.p, gr.p, n_enc, t, "decide-direct-carry-generator-litebullet", "litebullet-fold", true);
  out = {MatrixClaim<F>{gen.b_value, gen.b_point, msg.a_point}, EvalWithPoint<F>{msg.b_value, msg.b_point}};
  return true;
}

// ---------------------------------------------------------------- range audit
std::array<F, 2> GpuBackend::range_audit(const F& alpha, std::vector<uint64_t>& mult) {
  HostScope hs("range_audit");
  static std::mutex mu;
  static std::set<int> configured;
  int dev = 0;
  QF_CK(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!configured.count(dev)) {
      set_smem(qfd::k_range_audit, qfd::kAuditSmem);
      configured.insert(dev);
    }
  }
  // A warp's int8 counters are 32-bit: each warp takes at most
  // ceil(n / (16 * 512 * grid)) * 512 values of one launch.
  check(active_ < (uint64_t(1) << 40), "range audit: more than 2^40 values");
  qfd::AlphaPowers ap;
  F pw = alpha;
  for (int k = 0; k < qfd::kAuditGroup; ++k) {
    for (int j = 0; j < qfd::kC; ++j) ap.c[k][j] = uint32_t(pw.c[j]);
    pw = pw * alpha;
  }
  const unsigned grid = tile_grid(~uint64_t(0));  // one CTA per SM
  const size_t launches = src_ ? src_->live_blocks() : 1;
  DBuf<unsigned long long> hist(qfd::kAuditBins);
  DBuf<Fe> part(2 * size_t(grid) * std::max<size_t>(launches, 1));
  QF_CK(cudaMemsetAsync(hist.p, 0, hist.n * 8, s_));
  size_t li = 0;
  auto run = [&](const W* d, uint64_t n) {
    check(reinterpret_cast<uintptr_t>(d) % 16 == 0, "range audit: weights must be 16-byte aligned");
    QF_LAUNCH(s_, "k_range_audit", n * sizeof(W),
              qfd::k_range_audit<<<grid, qfd::kAuditThreads, qfd::kAuditSmem, s_>>>(d, n, ap, hist.p, part.p + 2 * size_t(grid) * li));
    ++li;
  };
  if (src_) src_->for_each(s_, [&](size_t, const W* d, uint64_t n) { run(d, n); });
  else if (active_) run(bva_, active_);
  mult.assign(qfd::kAuditBins, 0);
  std::vector<F> h(2 * size_t(grid) * li);
  QF_CK(cudaMemcpyAsync(mult.data(), hist.p, mult.size() * 8, cudaMemcpyDeviceToHost, s_));
  if (!h.empty()) QF_CK(cudaMemcpyAsync(h.data(), part.p, h.size() * 16, cudaMemcpyDeviceToHost, s_));
  QF_CK(cudaStreamSynchronize(s_));
  F num = F::zero(), den = F::one();
  for (size_t i = 0; i < h.size(); i += 2) {
    num = num * h[i + 1] + h[i] * den;
    den = den * h[i + 1];
  }
  return {num, den};
}

}  // namespace QFB_NS
