// Motion plans and base-level splitting; see geom.H for the reference
// behaviour each function reproduces.
#include "geom.H"

namespace cmg {

std::vector<Motion> exchangePlan(const Layout& g) {
  // Neighbours of box b are the other boxes meeting grow(b,1), in index order
  // (DisjointBoxLayout::computeNeighbors, BoxTools/DisjointBoxLayout.cpp:174-254).
  // An item is kept by trimEdges when its region touches a face ghost layer.
  std::vector<Motion> plan;
  const size_t n = g.size();
  for (size_t b = 0; b < n; ++b) {
    Box bghost = g[b].grow(1);
    for (size_t nb = 0; nb < n; ++nb) {
      if (nb == b) continue;
      const Box& nbox = g[nb];
      if (!bghost.intersects(nbox)) continue;
      Box region = nbox & bghost;
      bool keep = false;
      for (int d = 0; d < 3 && !keep; ++d) keep = g[b].grow(d, 1).intersects(region);
      if (keep) plan.push_back(Motion{(int)nb, (int)b, region, region});
    }
  }
  return plan;
}

std::vector<Motion> copyPlan(const Layout& src, const Layout& dst) {
  std::vector<Motion> plan;
  for (size_t d = 0; d < dst.size(); ++d)
    for (size_t s = 0; s < src.size(); ++s)
      if (dst[d].intersects(src[s])) {
        Box r = dst[d] & src[s];
        plan.push_back(Motion{(int)s, (int)d, r, r});
      }
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
