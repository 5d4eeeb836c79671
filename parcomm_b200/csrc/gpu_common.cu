// Field-independent CUDA infrastructure (see gpu_common.cuh).
#include "gpu_common.cuh"

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <thread>

namespace qfg {

namespace {
std::mutex g_pool_mu;
std::multimap<std::pair<int, size_t>, void*> g_pool;  // (device, rounded bytes) -> free device block
size_t g_pool_bytes = 0;                               // cached, all devices
size_t g_pool_limit = ~size_t(0);
int current_device() {
  int d = 0;
  QF_CK(cudaGetDevice(&d));
  return d;
}
}  // namespace

void* DevicePool::get(size_t bytes) {
  const size_t r = rounded(bytes);
  const int dev = current_device();
  {
    std::lock_guard<std::mutex> g(g_pool_mu);
    auto it = g_pool.find({dev, r});
    if (it != g_pool.end()) {
      void* p = it->second;
      g_pool.erase(it);
      g_pool_bytes -= r;
      return p;
    }
  }
  // On failure: free this device's cached blocks, largest first, only until
  // the request fits (the rest stays cached for the allocations that follow);
  // then, for up to half a second, wait for buffers that concurrent work is
  // about to release.
  void* p = nullptr;
  for (int waits = 0;;) {
    const cudaError_t e = cudaMalloc(&p, r);
    if (e == cudaSuccess) return p;
    cudaGetLastError();
    if (evict_one()) continue;
    if (++waits > 100) QF_CK(e);
    std::this_thread::sleep_for(std::chrono::milliseconds(5));
  }
}
// Frees the current device's largest cached block; false when none is left.
bool DevicePool::evict_one() {
  const int dev = current_device();
  std::lock_guard<std::mutex> g(g_pool_mu);
  auto best = g_pool.end();
  for (auto it = g_pool.begin(); it != g_pool.end(); ++it)
    if (it->first.first == dev && (best == g_pool.end() || it->first.second > best->first.second)) best = it;
  if (best == g_pool.end()) return false;
  cudaDeviceSynchronize();
  cudaFree(best->second);
  g_pool_bytes -= best->first.second;
  g_pool.erase(best);
  return true;
}
void DevicePool::put(void* p, size_t bytes) {
  const int dev = current_device();
  const size_t r = rounded(bytes);
  {
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (g_pool_bytes + r <= g_pool_limit) {
      g_pool.emplace(std::make_pair(dev, r), p);
      g_pool_bytes += r;
      return;
    }
  }
  cudaFree(p);  // over the cache limit
}
void DevicePool::set_limit(size_t bytes) {
  {
    std::lock_guard<std::mutex> g(g_pool_mu);
    g_pool_limit = bytes;
  }
  if (cached_bytes() > bytes) trim();
}
// Frees the current device's cached blocks.
void DevicePool::trim() {
  const int dev = current_device();
  std::lock_guard<std::mutex> g(g_pool_mu);
  cudaDeviceSynchronize();
  for (auto it = g_pool.begin(); it != g_pool.end();) {
    if (it->first.first == dev) {
      cudaFree(it->second);
      g_pool_bytes -= it->first.second;
      it = g_pool.erase(it);
    } else {
      ++it;
    }
  }
}
PinnedStage::Lease PinnedStage::acquire(size_t bytes) {
  static std::mutex mu;
  static void* buf = nullptr;
  static size_t cap = 0;
  Lease l{std::unique_lock<std::mutex>(mu), nullptr};
  if (bytes > cap) {
    if (buf) QF_CK(cudaFreeHost(buf));
    buf = nullptr;
    cap = 0;
    QF_CK(cudaHostAlloc(&buf, bytes, cudaHostAllocPortable));
    cap = bytes;
  }
  l.p = buf;
  return l;
}

size_t DevicePool::cached_bytes() {
  const int dev = current_device();
  std::lock_guard<std::mutex> g(g_pool_mu);
  size_t n = 0;
  for (auto& [k, p] : g_pool)
    if (k.first == dev) n += k.second;
  return n;
}

std::atomic<int> KernelOptions::imma{0};
std::atomic<int> KernelOptions::per_matrix{0};
std::atomic<int> KernelOptions::core_dots{0};

bool KernelClock::enabled = false;
std::mutex KernelClock::mu;
std::vector<KernelClock::Rec> KernelClock::recs;
std::atomic<uint64_t> KernelClock::launches{0};

KernelClock::Scope::Scope(cudaStream_t s, const char* n, uint64_t b_, uint64_t o_) : stream(s), name(n), bytes(b_), ops(o_) {
  if (enabled) {
    QF_CK(cudaEventCreate(&a));
    QF_CK(cudaEventCreate(&b));
    QF_CK(cudaEventRecord(a, stream));
  }
}
void KernelClock::Scope::done() {
  ++launches;
  if (enabled) {
    QF_CK(cudaEventRecord(b, stream));
    std::lock_guard<std::mutex> g(mu);
    recs.push_back({name, a, b, bytes, ops});
  }
}
void KernelClock::reset(bool on) {
  std::lock_guard<std::mutex> g(mu);
  for (auto& r : recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  recs.clear();
  ::qf::Sections::reset(on);
  enabled = on;
}
namespace {
std::mutex g_notes_mu;
std::map<std::string, std::string> g_notes;
}  // namespace
void KernelClock::note(const std::string& key, const std::string& json_value) {
  std::lock_guard<std::mutex> g(g_notes_mu);
  g_notes[key] = json_value;
}

std::string KernelClock::stats_json() {
  QF_CK(cudaDeviceSynchronize());
  std::lock_guard<std::mutex> g(mu);
  struct Agg { uint64_t n = 0, bytes = 0, ops = 0; double ms = 0; };
  std::map<std::string, Agg> agg;
  for (auto& r : recs) {
    float ms = 0;
    QF_CK(cudaEventElapsedTime(&ms, r.a, r.b));
    auto& e = agg[r.name];
    e.n += 1;
    e.ms += ms;
    e.bytes += r.bytes;
    e.ops += r.ops;
  }
  std::string s = "{";
  bool first = true;
  for (auto& [k, v] : agg) {
    if (!first) s += ",";
    first = false;
    char buf[256];
    std::snprintf(buf, sizeof buf, "\"%s\":{\"launches\":%llu,\"ms\":%.6f,\"bytes\":%llu,\"ops\":%llu}", k.c_str(),
                  (unsigned long long)v.n, v.ms, (unsigned long long)v.bytes, (unsigned long long)v.ops);
    s += buf;
  }
  // Idle time between consecutive recorded launches (in launch order), with
  // the largest gaps named by the kernels on either side.
  if (recs.size() > 1) {
    struct Gap { double ms; const char* before; const char* after; };
    std::vector<Gap> gaps;
    double total = 0;
    for (size_t i = 1; i < recs.size(); ++i) {
      float ms = 0;
      QF_CK(cudaEventElapsedTime(&ms, recs[i - 1].b, recs[i].a));
      if (ms > 0) { gaps.push_back({ms, recs[i - 1].name, recs[i].name}); total += ms; }
    }
    std::sort(gaps.begin(), gaps.end(), [](const Gap& x, const Gap& y) { return x.ms > y.ms; });
    if (!first) s += ",";
    first = false;
    char buf[256];
    std::snprintf(buf, sizeof buf, "\"_gaps\":{\"launches\":%llu,\"ms\":%.6f,\"bytes\":0,\"top\":[", (unsigned long long)gaps.size(), total);
    s += buf;
    for (size_t i = 0; i < gaps.size() && i < 40; ++i) {
      std::snprintf(buf, sizeof buf, "%s[\"%s\",\"%s\",%.4f]", i ? "," : "", gaps[i].before, gaps[i].after, gaps[i].ms);
      s += buf;
    }
    s += "]}";
  }
  std::lock_guard<std::mutex> gs(::qf::Sections::mu);
  for (auto& [k, v] : ::qf::Sections::totals) {
    if (!first) s += ",";
    first = false;
    char buf[256];
    std::snprintf(buf, sizeof buf, "\"host:%s\":{\"launches\":%llu,\"ms\":%.6f,\"bytes\":0}", k.c_str(),
                  (unsigned long long)v.first, v.second);
    s += buf;
  }
  std::lock_guard<std::mutex> gn(g_notes_mu);
  if (!g_notes.empty()) {
    if (!first) s += ",";
    first = false;
    s += "\"_notes\":{";
    bool f2 = true;
    for (auto& [k, v] : g_notes) {
      s += (f2 ? "\"" : ",\"") + k + "\":" + v;
      f2 = false;
    }
    s += "}";
  }
  return s + "}";
}

qfd::LeafPrefix leaf_prefix(size_t n_cols, bool ext_domain) {
  std::vector<uint8_t> pre;
  const char* dom = ext_domain ? kLeafExtDomain : kLeafBaseDomain;
  append_frame(pre, "domain", dom, std::strlen(dom));
  auto w = le64(n_cols);
  append_frame(pre, "width", w.data(), 8);
  if (pre.size() != (ext_domain ? 80u : 75u)) fail(QF_E_ENCODING, "leaf prefix length");
  qfd::LeafPrefix lp;
  uint32_t h[8];
  for (int i = 0; i < 8; ++i) h[i] = kBlake2sIv[i];
  h[0] ^= 0x01010000u ^ 32u;
  blake2s_compress(h, pre.data(), 64, false);
  for (int i = 0; i < 8; ++i) lp.mid[i] = h[i];
  uint8_t tail[16] = {0};
  std::memcpy(tail, pre.data() + 64, pre.size() - 64);
  for (int i = 0; i < 4; ++i)
    lp.tail[i] = uint32_t(tail[4 * i]) | (uint32_t(tail[4 * i + 1]) << 8) | (uint32_t(tail[4 * i + 2]) << 16) |
                 (uint32_t(tail[4 * i + 3]) << 24);
  return lp;
}
qfd::InnerPrefix inner_prefix() {
  std::vector<uint8_t> pre;
  append_frame(pre, "domain", kInnerDomain, std::strlen(kInnerDomain));
  if (pre.size() != 50) fail(QF_E_ENCODING, "inner prefix length");
  uint8_t b[52] = {0};
  std::memcpy(b, pre.data(), 50);
  qfd::InnerPrefix ip;
  for (int i = 0; i < 13; ++i)
    ip.w[i] = uint32_t(b[4 * i]) | (uint32_t(b[4 * i + 1]) << 8) | (uint32_t(b[4 * i + 2]) << 16) | (uint32_t(b[4 * i + 3]) << 24);
  return ip;
}


}  // namespace qfg
