// ORACLE (test infrastructure only): a range-splitting helper for the oracle's bulk loops.
//
// The reference runs single-threaded (its README prescribes one thread and the p3 `parallel`
// feature off).  The loops split here are the ones whose iterations are independent in the
// reference too: per-row DFTs and per-column hashes of `commit` (pcs/src/ligesis.rs:288-313),
// the column-wise GEMV of `prove` (:372-379), the per-pair sums of a sumcheck round
// (utils/src/sumcheck.rs:53-64) and Basefold's per-chunk DFTs and leaf hashes
// (pcs/src/basefold.rs:257-307).  Every result is an exact residue mod p, so splitting a sum
// into per-thread partial sums and adding them afterwards gives the same field element, and
// the oracle's outputs do not depend on the thread count.  The default is one thread; tests
// and bench.py's CPU leg raise it through orc_set_threads().
#pragma once
#include <algorithm>
#include <cstddef>
#include <exception>
#include <thread>
#include <vector>

namespace orc {

inline unsigned& oracle_threads() {
  static unsigned t = 1;
  return t;
}
// Set inside a worker: loops nested in a split loop run on that worker alone.
inline bool& oracle_in_worker() {
  thread_local bool w = false;
  return w;
}

// Number of ranges the helpers below use for n iterations with at least `grain` each.
inline size_t parallel_parts(size_t n, size_t grain = 1) {
  if (oracle_in_worker()) return 1;
  size_t parts = std::min<size_t>(oracle_threads(), grain ? (n + grain - 1) / grain : n);
  return parts ? parts : 1;
}

// Calls body(part, lo, hi) on parallel_parts(n, grain) disjoint ranges covering [0, n), one
// per thread, part = 0, 1, ... in range order.  The first exception thrown by any range is
// rethrown on the calling thread after every range has finished.
template <class F>
inline void parallel_chunks(size_t n, size_t grain, F&& body) {
  if (!n) return;
  size_t parts = parallel_parts(n, grain);
  if (parts <= 1) {
    body(size_t(0), size_t(0), n);
    return;
  }
  std::vector<std::thread> pool;
  std::vector<std::exception_ptr> errs(parts);
  size_t step = (n + parts - 1) / parts;
  for (size_t p = 0; p < parts; ++p) {
    size_t lo = p * step, hi = std::min(n, lo + step);
    if (lo >= hi) break;
    pool.emplace_back([&, p, lo, hi] {
      oracle_in_worker() = true;
      try {
        body(p, lo, hi);
      } catch (...) {
        errs[p] = std::current_exception();
      }
    });
  }
  for (auto& th : pool) th.join();
  for (auto& e : errs)
    if (e) std::rethrow_exception(e);
}

// body(lo, hi) over disjoint ranges of [0, n).
template <class F>
inline void parallel_ranges(size_t n, F&& body, size_t grain = 1) {
  parallel_chunks(n, grain, [&](size_t, size_t lo, size_t hi) { body(lo, hi); });
}

}  // namespace orc
