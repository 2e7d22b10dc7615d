// Checks of the kept large host blocks (hostmem.*): small requests are not
// kept, a freed block is handed to the next request that it fits (at most
// twice its size), the kept bytes stay within the cap, release empties the
// store, and concurrent allocations and frees from many threads keep every
// block distinct and the accounting exact.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <thread>
#include <vector>
#include "hostmem.H"
using namespace cmg;
#define CHECK(c)                                                   \
  do {                                                             \
    if (!(c)) {                                                    \
      std::fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); \
      return 1;                                                    \
    }                                                              \
  } while (0)
int main() {
  const size_t MiB = size_t(1) << 20;
  hostBlockRelease();
  CHECK(hostBlockKept() == 0);
  CHECK(hostBlockCap() > 0);
  // small blocks go straight back to the system
  void* s = hostBlockAlloc(1000);
  std::memset(s, 1, 1000);
  hostBlockFree(s, 1000);
  CHECK(hostBlockKept() == 0);
  // a 3 MiB block is kept (rounded to whole MiB) and reused for 2.5 MiB
  void* a = hostBlockAlloc(3 * MiB);
  std::memset(a, 2, 3 * MiB);
  hostBlockFree(a, 3 * MiB);
  CHECK(hostBlockKept() == 3 * MiB);
  void* b = hostBlockAlloc(5 * MiB / 2);
  CHECK(b == a);
  CHECK(hostBlockKept() == 0);
  std::memset(b, 3, 5 * MiB / 2);
  // freed with the size asked for, it is kept at its full 3 MiB
  hostBlockFree(b, 5 * MiB / 2);
  CHECK(hostBlockKept() == 3 * MiB);
  // not reused for a request of less than half its size
  void* c = hostBlockAlloc(MiB);
  CHECK(c != a);
  CHECK(hostBlockKept() == 3 * MiB);
  hostBlockFree(c, MiB);
  CHECK(hostBlockKept() == 4 * MiB);
  // nor for a larger one
  void* d = hostBlockAlloc(4 * MiB);
  CHECK(d != a && d != c);
  hostBlockFree(d, 4 * MiB);
  CHECK(hostBlockKept() == 8 * MiB);
  hostBlockRelease();
  CHECK(hostBlockKept() == 0);
  // many threads: every live block distinct, all kept after the frees
  const int T = 8, N = 40;
  std::vector<std::vector<void*>> got(T);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t]() {
      for (int i = 0; i < N; ++i) {
        const size_t n = (size_t)(1 + (t + i) % 3) * MiB;
        void* p = hostBlockAlloc(n);
        std::memset(p, t, n);
        got[t].push_back(p);
        if (i % 2) {
          hostBlockFree(got[t].front(), (size_t)(1 + t % 3) * MiB);
          got[t].erase(got[t].begin());
        }
      }
    });
  for (auto& x : th) x.join();
  std::set<void*> live;
  for (auto& v : got)
    for (void* p : v) live.insert(p);
  CHECK(live.size() == (size_t)T * N / 2);
  // every block freed (with any size of 1 MiB or more: the store knows each
  // block's own) is kept, up to the cap
  for (auto& v : got)
    for (void* p : v) hostBlockFree(p, MiB);
  CHECK(hostBlockKept() >= live.size() * MiB && hostBlockKept() <= hostBlockCap());
  hostBlockRelease();
  CHECK(hostBlockKept() == 0);
  std::printf("hostmem ok\n");
  return 0;
}
