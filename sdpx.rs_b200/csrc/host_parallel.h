// Static-chunk parallel loops for the host-side preprocessing of a prepare (input validation,
// Ruiz equilibration, operator packing): plain std::thread, no pool state between calls.
#pragma once
#include <algorithm>
#include <cstdint>
#include <exception>
#include <thread>
#include <vector>

namespace sdpxg {

inline int host_threads() {
  const unsigned hw = std::thread::hardware_concurrency();
  return (int)std::max(1u, std::min(hw, 32u));
}

// f(begin, end, chunk) over [0, n) split into at most host_threads() chunks of >= grain
// indices.  An exception thrown by any chunk is rethrown on the caller after all joined.
template <typename F>
void parallel_for(int64_t n, int64_t grain, F&& f) {
  const int64_t t = std::min<int64_t>(host_threads(), (n + grain - 1) / std::max<int64_t>(grain, 1));
  if (t <= 1) {
    if (n > 0) f(int64_t(0), n, 0);
    return;
  }
  std::vector<std::thread> th;
  std::vector<std::exception_ptr> err((size_t)t);
  th.reserve((size_t)t);
  for (int64_t i = 0; i < t; ++i)
    th.emplace_back([&, i] {
      try {
        f(n * i / t, n * (i + 1) / t, (int)i);
      } catch (...) {
        err[(size_t)i] = std::current_exception();
      }
    });
  for (auto& x : th) x.join();
  for (auto& e : err)
    if (e) std::rethrow_exception(e);
}

// Column grain for loops over the columns of a sparse matrix: chunks of at least ~64k stored
// entries, so small problems (many of them solved concurrently from separate host threads)
// stay on the calling thread instead of spawning threads for microseconds of work.
inline int64_t col_grain(uint64_t cols, uint64_t nnz) {
  if (cols == 0) return 1;
  const double per_col = std::max(1.0, (double)nnz / (double)cols);
  return std::max<int64_t>(8, (int64_t)(65536.0 / per_col));
}

}  // namespace sdpxg
