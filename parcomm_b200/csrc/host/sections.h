// Named host wall-clock sections.  Recording is off by default; the
// library's per-kernel timing switch turns it on, and the totals are reported
// beside the kernel times as "host:<name>".
#pragma once
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <utility>

namespace qf {

struct Sections {
  static inline std::atomic<bool> enabled{false};
  static inline std::mutex mu;
  static inline std::map<std::string, std::pair<uint64_t, double>> totals;  // name -> (count, ms)
  static void reset(bool on) {
    std::lock_guard<std::mutex> g(mu);
    totals.clear();
    enabled = on;
  }
};

struct Section {
  const char* name;
  bool on;
  std::chrono::steady_clock::time_point t0;
  explicit Section(const char* n) : name(n), on(Sections::enabled.load()) {
    if (on) t0 = std::chrono::steady_clock::now();
  }
  ~Section() {
    if (!on) return;
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> g(Sections::mu);
    auto& e = Sections::totals[name];
    e.first += 1;
    e.second += ms;
  }
  Section(const Section&) = delete;
  Section& operator=(const Section&) = delete;
};

}  // namespace qf
