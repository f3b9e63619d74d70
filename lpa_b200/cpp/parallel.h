// Minimal host thread pool helpers for the format layer (std::thread only).
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

namespace lpa {

inline int resolve_threads(int threads) {
  if (threads > 0) return threads;
  unsigned h = std::thread::hardware_concurrency();
  return h ? static_cast<int>(h) : 1;
}

// Runs fn(begin, end, tid) over [0, n) in chunks of `grain`, dynamically
// scheduled over `threads` workers.
template <class Fn>
void parallel_for(uint64_t n, uint64_t grain, int threads, Fn fn) {
  threads = resolve_threads(threads);
  if (n == 0) return;
  if (grain == 0) grain = 1;
  uint64_t chunks = (n + grain - 1) / grain;
  if (threads <= 1 || chunks <= 1) {
    fn(uint64_t(0), n, 0);
    return;
  }
  int nt = static_cast<int>(std::min<uint64_t>(static_cast<uint64_t>(threads), chunks));
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> pool;
  pool.reserve(nt);
  for (int t = 0; t < nt; t++) {
    pool.emplace_back([&, t]() {
      for (;;) {
        uint64_t c = next.fetch_add(1, std::memory_order_relaxed);
        if (c >= chunks) break;
        uint64_t b = c * grain, e = std::min(n, b + grain);
        fn(b, e, t);
      }
    });
  }
  for (auto &th : pool) th.join();
}

// Static partition: fn(begin, end, tid) once per worker over contiguous ranges.
template <class Fn>
void parallel_ranges(uint64_t n, int threads, Fn fn) {
  threads = resolve_threads(threads);
  if (n == 0) return;
  int nt = static_cast<int>(std::min<uint64_t>(static_cast<uint64_t>(threads), n));
  if (nt <= 1) {
    fn(uint64_t(0), n, 0);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; t++) {
    uint64_t b = n * t / nt, e = n * (t + 1) / nt;
    pool.emplace_back([=]() { fn(b, e, t); });
  }
  for (auto &th : pool) th.join();
}

}  // namespace lpa
