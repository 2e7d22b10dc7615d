// Index-space calculus for the AMR elliptic solve: integer vectors, cell
// boxes, dense cell sets and box layouts.  Semantics follow the reference's
// BoxTools so that every layout, motion plan and coarse-fine set built from
// them matches the reference bit for bit:
//   IntVect lexical order (x, then y, then z)  BoxTools/IntVect.H:898-915
//   Box order (smallEnd lexical, then bigEnd)  BoxTools/Box.H:2221-2225
//   coarsen = floor division                    BoxTools/IntVect.H (coarsen)
// Only cell-centred boxes in 3D are needed on this path; face-centred data
// is addressed through cell boxes plus a direction.
#ifndef CMG_GEOM_H
#define CMG_GEOM_H

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

namespace cmg {

struct IV {
  int v[3];
  IV() : v{0, 0, 0} {}
  IV(int a, int b, int c) : v{a, b, c} {}
  int& operator[](int d) { return v[d]; }
  int operator[](int d) const { return v[d]; }
  bool operator==(const IV& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
  bool operator!=(const IV& o) const { return !(*this == o); }
  bool lexLT(const IV& o) const {
    if (v[0] != o.v[0]) return v[0] < o.v[0];
    if (v[1] != o.v[1]) return v[1] < o.v[1];
    return v[2] < o.v[2];
  }
  IV operator+(const IV& o) const { return IV(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]); }
  IV operator-(const IV& o) const { return IV(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]); }
  static IV basis(int d, int s = 1) {
    IV r;
    r.v[d] = s;
    return r;
  }
};

inline int floordiv(int a, int r) { return a >= 0 ? a / r : -((-a + r - 1) / r); }

struct Box {
  IV lo, hi;  // inclusive; empty when any hi < lo
  Box() : lo(0, 0, 0), hi(-1, -1, -1) {}
  Box(const IV& l, const IV& h) : lo(l), hi(h) {}
  bool empty() const { return hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2]; }
  int size(int d) const { return hi[d] - lo[d] + 1; }
  int64_t numPts() const { return empty() ? 0 : (int64_t)size(0) * size(1) * size(2); }
  bool contains(const IV& p) const {
    return p[0] >= lo[0] && p[0] <= hi[0] && p[1] >= lo[1] && p[1] <= hi[1] && p[2] >= lo[2] &&
           p[2] <= hi[2];
  }
  bool contains(const Box& b) const { return b.empty() || (contains(b.lo) && contains(b.hi)); }
  bool intersects(const Box& b) const {
    for (int d = 0; d < 3; ++d)
      if (std::max(lo[d], b.lo[d]) > std::min(hi[d], b.hi[d])) return false;
    return !empty() && !b.empty();
  }
  Box operator&(const Box& b) const {
    Box r;
    for (int d = 0; d < 3; ++d) {
      r.lo[d] = std::max(lo[d], b.lo[d]);
      r.hi[d] = std::min(hi[d], b.hi[d]);
    }
    return r;
  }
  bool operator==(const Box& b) const { return lo == b.lo && hi == b.hi; }
  bool operator!=(const Box& b) const { return !(*this == b); }
  // Box.H:2221-2225 ordering.
  bool operator<(const Box& r) const {
    if (lo == r.lo) return hi.lexLT(r.hi);
    return !empty() && (r.empty() || lo.lexLT(r.lo));
  }
  Box grow(int n) const { return Box(lo - IV(n, n, n), hi + IV(n, n, n)); }
  Box grow(int d, int n) const {
    Box r = *this;
    r.lo[d] -= n;
    r.hi[d] += n;
    return r;
  }
  Box shift(int d, int n) const {
    Box r = *this;
    r.lo[d] += n;
    r.hi[d] += n;
    return r;
  }
  Box shift(const IV& s) const { return Box(lo + s, hi + s); }
  Box coarsen(int r) const {
    Box b;
    for (int d = 0; d < 3; ++d) {
      b.lo[d] = floordiv(lo[d], r);
      b.hi[d] = floordiv(hi[d], r);
    }
    return b;
  }
  Box refine(int r) const {
    Box b;
    for (int d = 0; d < 3; ++d) {
      b.lo[d] = lo[d] * r;
      b.hi[d] = hi[d] * r + r - 1;
    }
    return b;
  }
  bool coarsenable(int r) const { return coarsen(r).refine(r) == *this; }
  // Cells adjacent to the low (side -1) or high (side +1) face, n deep.
  Box adjCell(int d, int side, int n) const {
    Box r = *this;
    if (side < 0) {
      r.hi[d] = lo[d] - 1;
      r.lo[d] = lo[d] - n;
    } else {
      r.lo[d] = hi[d] + 1;
      r.hi[d] = hi[d] + n;
    }
    return r;
  }
};

// Dense cell set over a bounding box, the subset of IntVectSet semantics the
// coarse-fine set construction needs (BoxTools/DenseIntVectSet.cpp).
struct CellSet {
  Box dom;
  std::vector<uint8_t> bits;
  CellSet() {}
  explicit CellSet(const Box& b, bool val = true) { define(b, val); }
  void define(const Box& b, bool val = true) {
    dom = b;
    bits.assign(b.empty() ? 0 : (size_t)b.numPts(), val ? 1 : 0);
  }
  size_t at(const IV& p) const {
    return (size_t)(p[0] - dom.lo[0]) +
           (size_t)dom.size(0) * ((size_t)(p[1] - dom.lo[1]) + (size_t)dom.size(1) * (p[2] - dom.lo[2]));
  }
  bool contains(const IV& p) const { return dom.contains(p) && bits[at(p)]; }
  bool containsBox(const Box& b) const {
    if (b.empty()) return true;
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
      for (int j = b.lo[1]; j <= b.hi[1]; ++j)
        for (int i = b.lo[0]; i <= b.hi[0]; ++i)
          if (!contains(IV(i, j, k))) return false;
    return true;
  }
  void set(const Box& b, bool val) {
    Box c = b & dom;
    if (c.empty()) return;
    for (int k = c.lo[2]; k <= c.hi[2]; ++k)
      for (int j = c.lo[1]; j <= c.hi[1]; ++j)
        for (int i = c.lo[0]; i <= c.hi[0]; ++i) bits[at(IV(i, j, k))] = val ? 1 : 0;
  }
  void subtract(const Box& b) { set(b, false); }
  void intersect(const Box& b) {
    if (dom.empty() || (b.contains(dom.lo) && b.contains(dom.hi))) return;
    for (int k = dom.lo[2]; k <= dom.hi[2]; ++k)
      for (int j = dom.lo[1]; j <= dom.hi[1]; ++j)
        for (int i = dom.lo[0]; i <= dom.hi[0]; ++i)
          if (!b.contains(IV(i, j, k))) bits[at(IV(i, j, k))] = 0;
  }
  int64_t numPts() const {
    int64_t n = 0;
    for (uint8_t b : bits) n += b;
    return n;
  }
  bool empty() const { return std::find(bits.begin(), bits.end(), (uint8_t)1) == bits.end(); }
  Box minBox() const {
    Box r;
    bool first = true;
    for (int k = dom.lo[2]; k <= dom.hi[2]; ++k)
      for (int j = dom.lo[1]; j <= dom.hi[1]; ++j)
        for (int i = dom.lo[0]; i <= dom.hi[0]; ++i)
          if (bits[at(IV(i, j, k))]) {
            IV p(i, j, k);
            if (first) {
              r = Box(p, p);
              first = false;
            } else
              for (int d = 0; d < 3; ++d) {
                r.lo[d] = std::min(r.lo[d], p[d]);
                r.hi[d] = std::max(r.hi[d], p[d]);
              }
          }
    return r;
  }
  // Members in x-fastest order.
  std::vector<IV> cells() const {
    std::vector<IV> out;
    for (int k = dom.lo[2]; k <= dom.hi[2]; ++k)
      for (int j = dom.lo[1]; j <= dom.hi[1]; ++j)
        for (int i = dom.lo[0]; i <= dom.hi[0]; ++i)
          if (bits[at(IV(i, j, k))]) out.push_back(IV(i, j, k));
    return out;
  }
  CellSet coarsen(int r) const {
    CellSet c(dom.coarsen(r), false);
    for (const IV& p : cells()) c.bits[c.at(IV(floordiv(p[0], r), floordiv(p[1], r), floordiv(p[2], r)))] = 1;
    return c;
  }
  // Erosion along d by one cell (DenseIntVectSet::grow with a negative count).
  CellSet erode(int d) const {
    CellSet c(dom, false);
    for (const IV& p : cells())
      if (contains(p + IV::basis(d, 1)) && contains(p - IV::basis(d, 1))) c.bits[c.at(p)] = 1;
    return c;
  }
};

// A sorted, disjoint set of boxes on one level (DisjointBoxLayout after
// close(): BoxTools/BoxLayout.cpp:89-119).
struct Layout {
  std::vector<Box> boxes;
  Layout() {}
  explicit Layout(std::vector<Box> b) : boxes(std::move(b)) { std::sort(boxes.begin(), boxes.end()); }
  size_t size() const { return boxes.size(); }
  const Box& operator[](size_t i) const { return boxes[i]; }
  int64_t numCells() const {
    int64_t n = 0;
    for (auto& b : boxes) n += b.numPts();
    return n;
  }
  bool coarsenable(int r) const {
    for (auto& b : boxes)
      if (!b.coarsenable(r)) return false;
    return true;
  }
  // Box-wise coarsening keeps the index order (coarsen_dbl in the reference).
  Layout coarsen(int r) const {
    Layout l;
    for (auto& b : boxes) l.boxes.push_back(b.coarsen(r));
    return l;
  }
};

// One local copy of the reference's Copier (BoxTools/Copier.H:36-57).
struct Motion {
  int from, to;
  Box fromRegion, toRegion;
};

// Copier::exchangeDefine + trimEdges (BoxTools/Copier.cpp:1464-1516,142-177)
// for one ghost layer, non-periodic domain.
std::vector<Motion> exchangePlan(const Layout& g);
// The same with the periodic images of the domain in the directions where
// periodic[d] (fromRegion in the source box's own coordinates).
std::vector<Motion> exchangePlan(const Layout& g, const Box& domain, const bool* periodic);
// Copier::define(src, dest, ghost=0) local plan (BoxTools/Copier.cpp:903-1110).
std::vector<Motion> copyPlan(const Layout& src, const Layout& dst);
// Spatial index of a box list: the boxes overlapping each block of B^3
// cells, so that "every box meeting region r" costs the blocks of r instead
// of the whole list.  query() returns box indices in increasing order.
struct BoxIndex {
  int B = 8;
  IV org, n;
  std::vector<int> start, ids;  // CSR: blocks -> box indices
  void build(const std::vector<Box>& boxes, int blockSize = 8) {
    B = blockSize;
    start.clear();
    ids.clear();
    if (boxes.empty()) {
      n = IV(0, 0, 0);
      return;
    }
    Box all = boxes[0];
    for (const Box& b : boxes)
      for (int d = 0; d < 3; ++d) {
        all.lo[d] = std::min(all.lo[d], b.lo[d]);
        all.hi[d] = std::max(all.hi[d], b.hi[d]);
      }
    Box c = all.coarsen(B);
    org = c.lo;
    n = IV(c.size(0), c.size(1), c.size(2));
    const size_t nb = (size_t)n[0] * n[1] * n[2];
    std::vector<int> count(nb + 1, 0);
    auto each = [&](const Box& b, auto fn) {
      Box q = b.coarsen(B);
      for (int z = q.lo[2]; z <= q.hi[2]; ++z)
        for (int y = q.lo[1]; y <= q.hi[1]; ++y)
          for (int x = q.lo[0]; x <= q.hi[0]; ++x) fn(slot(IV(x, y, z)));
    };
    for (const Box& b : boxes) each(b, [&](size_t s) { count[s + 1]++; });
    for (size_t i = 0; i < nb; ++i) count[i + 1] += count[i];
    start = count;
    ids.assign(count[nb], 0);
    std::vector<int> fillp(count.begin(), count.end() - 1);
    for (size_t k = 0; k < boxes.size(); ++k) each(boxes[k], [&](size_t s) { ids[fillp[s]++] = (int)k; });
  }
  size_t slot(const IV& q) const {
    return (size_t)(q[0] - org[0]) + (size_t)n[0] * ((size_t)(q[1] - org[1]) + (size_t)n[1] * (q[2] - org[2]));
  }
  // Indices of the boxes of `boxes` that intersect r (increasing order).
  // Read-only, so concurrent queries are safe.
  void query(const std::vector<Box>& boxes, const Box& r, std::vector<int>& out) const {
    out.clear();
    if (r.empty() || n[0] == 0) return;
    Box q = r.coarsen(B);
    for (int z = std::max(q.lo[2], org[2]); z <= std::min(q.hi[2], org[2] + n[2] - 1); ++z)
      for (int y = std::max(q.lo[1], org[1]); y <= std::min(q.hi[1], org[1] + n[1] - 1); ++y)
        for (int x = std::max(q.lo[0], org[0]); x <= std::min(q.hi[0], org[0] + n[0] - 1); ++x) {
          size_t s = slot(IV(x, y, z));
          for (int i = start[s]; i < start[s + 1]; ++i)
            if (boxes[ids[i]].intersects(r)) out.push_back(ids[i]);
        }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
  }
};

// domainSplit (BoxTools/BRMeshRefine.cpp:983-1092) with all directions refined.
std::vector<Box> domainSplit(const Box& domain, int maxBoxSize, int blockFactor);

}  // namespace cmg

#endif
