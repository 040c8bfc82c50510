// Host-side parallel loop shared by the solvers' convergence tests.
#pragma once

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace tbgpu {

// true inside a parallel_for worker thread
inline bool &in_parallel_for() {
  thread_local bool flag = false;
  return flag;
}

// run f(i) for i in [0, n) on up to hardware_concurrency host threads; a
// parallel_for called from inside another one runs serially on its thread
template <class F>
inline void parallel_for(int n, F f) {
  int nt = int(std::thread::hardware_concurrency());
  nt = std::max(1, std::min({nt, 32, n}));
  if (nt <= 1 || in_parallel_for()) {
    for (int i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&]() {
      in_parallel_for() = true;
      for (int i = next++; i < n; i = next++) f(i);
    });
  for (auto &x : th) x.join();
}

}  // namespace tbgpu
