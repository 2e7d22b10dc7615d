// Host thread pool for the plan builders, grid generation and host-side
// fills: one set of worker threads per process, shared by every caller, so
// that concurrent requests (serving) and nested loops (levels built on their
// own threads, each looping over boxes) neither create threads per loop nor
// run more threads than the host has cores.
#ifndef CMG_HOSTPOOL_H
#define CMG_HOSTPOOL_H

#include <cstddef>
#include <functional>

namespace cmg {

// Runs fn(i) for every i in [0, n), the calling thread included, and returns
// when all have finished; items must write disjoint data (their order is
// not fixed).  The first exception an item throws is rethrown here once
// every item has ended.  Safe to call from inside an item.
void hostParallel(size_t n, const std::function<void(size_t)>& fn);

}  // namespace cmg

#endif
