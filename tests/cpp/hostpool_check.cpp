// Checks of the host thread pool (chombo_3.2_b200/csrc/hostpool.*): every
// item runs exactly once, nested and concurrent calls from many threads
// finish, and an item's exception reaches the caller after the other items.
#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <thread>
#include <vector>

#include "hostpool.H"

int main() {
  // every item exactly once
  std::vector<std::atomic<int>> hits(10000);
  for (auto& h : hits) h = 0;
  cmg::hostParallel(hits.size(), [&](size_t i) { hits[i]++; });
  for (auto& h : hits)
    if (h != 1) return 1;
  // nested calls from many threads at once
  std::atomic<long> sum{0};
  std::vector<std::thread> th;
  for (int t = 0; t < 24; ++t)
    th.emplace_back([&, t]() {
      for (int rep = 0; rep < 100; ++rep)
        cmg::hostParallel(17 + t, [&](size_t i) {
          cmg::hostParallel(5, [&](size_t j) { sum += (long)((i * 5 + j) % 7); });
        });
    });
  for (auto& x : th) x.join();
  long expect = 0;
  for (int t = 0; t < 24; ++t)
    for (int i = 0; i < 17 + t; ++i)
      for (int j = 0; j < 5; ++j) expect += 100 * ((i * 5 + j) % 7);
  if (sum != expect) return 2;
  // the first exception reaches the caller, after every other item ran
  std::atomic<int> ran{0};
  bool caught = false;
  try {
    cmg::hostParallel(200, [&](size_t i) {
      ran++;
      if (i == 57) throw std::runtime_error("item 57");
    });
  } catch (const std::runtime_error&) {
    caught = true;
  }
  if (!caught || ran != 200) return 3;
  // empty and single-item calls
  cmg::hostParallel(0, [&](size_t) { std::abort(); });
  int one = 0;
  cmg::hostParallel(1, [&](size_t) { one++; });
  if (one != 1) return 4;
  std::printf("hostpool ok\n");
  return 0;
}
