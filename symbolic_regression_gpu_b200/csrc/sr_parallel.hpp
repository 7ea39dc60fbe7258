// sr_parallel.hpp — minimal fork-join helper for host-side passes.
#pragma once
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace sr {

template <class F>
void parallel_for(int64_t n, int threads, F &&fn) {
  if (n <= 0) return;
  const int64_t t = std::max<int64_t>(1, std::min<int64_t>(threads, n));
  if (t == 1) {
    fn(int64_t{0}, n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(static_cast<size_t>(t - 1));
  for (int64_t k = 1; k < t; ++k)
    pool.emplace_back([&, k] { fn(n * k / t, n * (k + 1) / t); });
  fn(int64_t{0}, n / t);
  for (auto &th : pool) th.join();
}

}  // namespace sr
