// Motion plans and base-level splitting; see geom.H for the reference
// behaviour each function reproduces.
#include "geom.H"

#include "hostpool.H"

namespace cmg {

std::vector<Motion> exchangePlan(const Layout& g) { return exchangePlan(g, Box(), nullptr); }

std::vector<Motion> exchangePlan(const Layout& g, const Box& domain, const bool* periodic) {
  // Neighbours of box b are the other boxes meeting grow(b,1), in index order
  // (DisjointBoxLayout::computeNeighbors, BoxTools/DisjointBoxLayout.cpp:174-254),
  // found through a spatial index.  In a periodic direction the domain's
  // images shifted by +-its length are neighbours too, listed after the
  // direct ones by source box and then by shift, the shifts ordered with x
  // outermost (ShiftIterator::computeShifts, BoxTools/ProblemDomain.cpp:45-110):
  // their items copy from the source box at region - shift.  An item is kept
  // by trimEdges when its region touches a face ghost layer.
  std::vector<Motion> plan;
  const size_t n = g.size();
  std::vector<IV> shifts;
  if (periodic) {
    const int r[3] = {periodic[0] ? 1 : 0, periodic[1] ? 1 : 0, periodic[2] ? 1 : 0};
    for (int x = -r[0]; x <= r[0]; ++x)
      for (int y = -r[1]; y <= r[1]; ++y)
        for (int z = -r[2]; z <= r[2]; ++z)
          if (x || y || z) shifts.push_back(IV(x * domain.size(0), y * domain.size(1), z * domain.size(2)));
  }
  BoxIndex index;
  index.build(g.boxes);
  struct Image {
    int nb, shift;
    Motion m;
  };
  auto kept = [&](size_t b, const Box& region) {
    for (int d = 0; d < 3; ++d)
      if (g[b].grow(d, 1).intersects(region)) return true;
    return false;
  };
  // each box's items on a host thread, concatenated in box order
  std::vector<std::vector<Motion>> perBox(n);
  hostParallel(n, [&](size_t b) {
    std::vector<int> hits;
    std::vector<Image> images;
    std::vector<Motion>& out = perBox[b];
    const Box bghost = g[b].grow(1);
    index.query(g.boxes, bghost, hits);
    for (int nb : hits) {
      if (nb == (int)b) continue;
      const Box region = g[nb] & bghost;
      if (!region.empty() && kept(b, region)) out.push_back(Motion{nb, (int)b, region, region});
    }
    if (shifts.empty() || domain.contains(bghost)) return;
    for (size_t k = 0; k < shifts.size(); ++k) {
      const IV& sh = shifts[k];
      const IV back(-sh[0], -sh[1], -sh[2]);
      index.query(g.boxes, bghost.shift(back), hits);
      for (int nb : hits) {
        const Box region = g[nb].shift(sh) & bghost;
        if (!region.empty() && kept(b, region))
          images.push_back(Image{nb, (int)k, Motion{nb, (int)b, region.shift(back), region}});
      }
    }
    std::sort(images.begin(), images.end(),
              [](const Image& a, const Image& c) { return a.nb != c.nb ? a.nb < c.nb : a.shift < c.shift; });
    for (const Image& im : images) out.push_back(im.m);
  });
  size_t total = 0;
  for (const auto& v : perBox) total += v.size();
  plan.reserve(total);
  for (const auto& v : perBox) plan.insert(plan.end(), v.begin(), v.end());
  return plan;
}

std::vector<Motion> copyPlan(const Layout& src, const Layout& dst) {
  // per destination box, the source boxes meeting it in index order (through
  // a spatial index, on host threads), concatenated in destination order
  BoxIndex index;
  index.build(src.boxes);
  std::vector<std::vector<Motion>> perBox(dst.size());
  hostParallel(dst.size(), [&](size_t d) {
    std::vector<int> hits;
    index.query(src.boxes, dst[d], hits);
    for (int s : hits) {
      Box r = dst[d] & src[s];
      if (!r.empty()) perBox[d].push_back(Motion{s, (int)d, r, r});
    }
  });
  std::vector<Motion> plan;
  for (const auto& v : perBox) plan.insert(plan.end(), v.begin(), v.end());
  return plan;
}

std::vector<Box> domainSplit(const Box& domain, int maxBoxSize, int blockFactor) {
  std::vector<Box> out;
  if (maxBoxSize == 0) {
    out.push_back(domain);
    return out;
  }
  int ratio = maxBoxSize / blockFactor;
  Box d = domain.coarsen(blockFactor);
  if (d.refine(blockFactor) != domain) std::abort();
  size_t count[4] = {1, 0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    int c = (d.hi[i] - d.lo[i] + ratio) / ratio;
    count[i + 1] = count[i] * (size_t)c;
  }
  out.resize(count[3]);
  for (size_t b = 0; b < out.size(); ++b) {
    IV lo = d.lo, hi = d.hi;
    for (int i = 0; i < 3; ++i) {
      int m = (int)((b / count[i]) % (count[i + 1] / count[i]));
      lo[i] += m * ratio;
      hi[i] = std::min(d.hi[i], lo[i] + ratio - 1);
    }
    out[b] = Box(lo, hi).refine(blockFactor);
  }
  return out;
}

}  // namespace cmg
