// Minimal host parallel-for for the planning passes (pattern building, analysis
// maps): [0, n) is cut into one contiguous range per thread and f runs on each
// range; callers only use it where every index writes its own outputs, or merge
// per-range results in range order, so the result does not depend on the thread
// count.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <exception>
#include <thread>
#include <vector>

namespace tdem {

// host threads of the planning passes: TDEM_HOST_THREADS if set, else the
// hardware threads (at most 32)
inline int host_threads() {
  if (const char* v = std::getenv("TDEM_HOST_THREADS")) {
    const int t = std::atoi(v);
    if (t > 0) return std::min(t, 256);
  }
  const unsigned h = std::thread::hardware_concurrency();
  return (int)std::max(1u, std::min(h, 32u));
}

// number of ranges parallel_chunks cuts [0, n) into, at least min_per_thread each
inline int chunk_count(int64_t n, int64_t min_per_thread = 4096) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(host_threads(), n / std::max<int64_t>(1, min_per_thread)));
}

// f(t, begin, end) for the t-th of nt contiguous ranges of [0, n), range t on its own
// thread; an exception thrown by any range is rethrown here after all have ended
template <class F>
void parallel_chunks(int64_t n, int nt, F&& f) {
  nt = std::max(1, nt);
  const int64_t step = (n + nt - 1) / nt;
  std::vector<std::exception_ptr> err(nt);
  auto range = [&](int t) {
    try {
      const int64_t b = std::min(n, t * step), e = std::min(n, (t + 1) * step);
      f(t, b, e);
    } catch (...) {
      err[t] = std::current_exception();
    }
  };
  if (nt > 1) {
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    // a range whose thread cannot be started (std::system_error) runs inline on this
    // thread after the started ones, so every range runs once and every started
    // thread is joined before anything leaves this scope
    int started = 1;
    try {
      for (; started < nt; ++started) pool.emplace_back([&range, t = started] { range(t); });
    } catch (...) {
    }
    range(0);
    for (int t = started; t < nt; ++t) range(t);
    for (std::thread& th : pool) th.join();
  } else {
    range(0);
  }
  for (const std::exception_ptr& x : err)
    if (x) std::rethrow_exception(x);
}

template <class F>
void parallel_ranges(int64_t n, F&& f, int64_t min_per_thread = 4096) {
  parallel_chunks(n, chunk_count(n, min_per_thread), [&f](int, int64_t b, int64_t e) { f(b, e); });
}

}  // namespace tdem
