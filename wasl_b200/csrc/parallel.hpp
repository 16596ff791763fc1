// A minimal fork-join loop over the host's threads for setup work.
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace wasl_b200 {

// body(begin, end) over [0, n) split into contiguous ranges, one per host
// thread (a single call for small n).
template <typename F> void parallel_for(std::int64_t n, F &&body) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const std::int64_t workers = std::min<std::int64_t>(hw, std::max<std::int64_t>(1, n / 256));
  if (workers <= 1) {
    body(0, n);
    return;
  }
  std::vector<std::thread> pool;
  for (std::int64_t w = 0; w < workers; ++w)
    pool.emplace_back([&, w] { body(n * w / workers, n * (w + 1) / workers); });
  for (auto &t : pool)
    t.join();
}

} // namespace wasl_b200
