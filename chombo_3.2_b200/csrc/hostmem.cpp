#include "hostmem.H"

#include <unistd.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>

namespace cmg {

namespace {

constexpr size_t kBig = size_t(1) << 20;

struct Blocks {
  std::mutex m;
  std::multimap<size_t, void*> kept;       // size -> block
  std::unordered_map<void*, size_t> size;  // every large block handed out -> its size
  size_t keptBytes = 0;
  size_t cap = 0;
  Blocks() {
    const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
    const size_t phys = pages > 0 && page > 0 ? (size_t)pages * (size_t)page : 0;
    cap = std::min(size_t(8) << 30, phys / 8);
  }
};

Blocks& blocks() {
  static Blocks* b = new Blocks();  // never destroyed: tables may be freed during static destruction
  return *b;
}

}  // namespace

void* hostBlockAlloc(size_t bytes) {
  if (bytes < kBig) return ::operator new(bytes);
  const size_t r = (bytes + kBig - 1) & ~(kBig - 1);
  Blocks& B = blocks();
  {
    std::lock_guard<std::mutex> lk(B.m);
    auto it = B.kept.lower_bound(r);  // the smallest kept block that fits
    if (it != B.kept.end() && it->first / 2 <= r) {
      void* p = it->second;
      B.keptBytes -= it->first;
      B.size[p] = it->first;
      B.kept.erase(it);
      return p;
    }
  }
  void* p = ::operator new(r);
  std::lock_guard<std::mutex> lk(B.m);
  B.size[p] = r;
  return p;
}

void hostBlockFree(void* p, size_t bytes) {
  if (!p) return;
  if (bytes < kBig) {
    ::operator delete(p);
    return;
  }
  Blocks& B = blocks();
  std::unique_lock<std::mutex> lk(B.m);
  auto it = B.size.find(p);
  const size_t r = it != B.size.end() ? it->second : 0;
  if (it != B.size.end()) B.size.erase(it);
  if (r && B.keptBytes + r <= B.cap) {
    B.kept.emplace(r, p);
    B.keptBytes += r;
    return;
  }
  lk.unlock();
  ::operator delete(p);
}

size_t hostBlockKept() {
  Blocks& B = blocks();
  std::lock_guard<std::mutex> lk(B.m);
  return B.keptBytes;
}

size_t hostBlockCap() { return blocks().cap; }

void hostBlockRelease() {
  Blocks& B = blocks();
  std::multimap<size_t, void*> out;
  {
    std::lock_guard<std::mutex> lk(B.m);
    out.swap(B.kept);
    B.keptBytes = 0;
  }
  for (auto& kv : out) ::operator delete(kv.second);
}

}  // namespace cmg
