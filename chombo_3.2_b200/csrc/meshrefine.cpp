// Grid generation: MeshRefine::regrid + BRMeshRefine::makeBoxes (see
// meshrefine.H).  Cell sets are dense bitmaps over a level's domain (the
// reference uses IntVectSet; only set membership, counts and tight bounding
// boxes enter the algorithm, so the representation does not change the
// result).
#include "meshrefine.H"

#include "hostpool.H"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <thread>

#include "synthetic.H"

namespace cmg {

namespace {

// BRMeshRefine.cpp: _BR_MIN_INFLECTION_MAG_
constexpr int kMinInflectionMag = 3;

bool isPow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// BRMeshRefine::longsideRefineDirs (BRMeshRefine.cpp:1202-1220): the
// longest side, the lowest direction on ties.
int longside(const Box& b, int& dir) {
  int maxlen = b.size(0);
  dir = 0;
  for (int d = 1; d < 3; ++d)
    if (b.size(d) > maxlen) {
      maxlen = b.size(d);
      dir = d;
    }
  return maxlen;
}

// BRMeshRefine::findSplit (BRMeshRefine.cpp:694-753): a zero of the trace,
// searched outward from the middle when the trace is longer than twice the
// maximum box size, else the first interior one.
int findSplit(const std::vector<int>& tr, int maxBoxSize) {
  const int n = (int)tr.size();
  if (n > 2 * maxBoxSize) {
    int iforward = n / 2 + 1;
    for (int i = n / 2; i >= 1 && iforward < n - 1; --i, ++iforward) {
      if (tr[i] == 0) return i;
      if (tr[iforward] == 0) return iforward;
    }
    return -1;
  }
  for (int i = 1; i < n - 1; ++i)
    if (tr[i] == 0) return i;
  return -1;
}

// BRMeshRefine::findMaxInflectionPoint (BRMeshRefine.cpp:755-863): the
// strongest sign change of the trace's second difference (at least
// kMinInflectionMag), searched the same way as findSplit.
int findInflection(const std::vector<int>& tr, int maxBoxSize) {
  const int n = (int)tr.size();
  std::vector<int> d2(n, 0);
  for (int i = 1; i < n - 1; ++i) d2[i] = tr[i - 1] - 2 * tr[i] + tr[i + 1];
  int imax = 0, maxVal = -1;
  auto test = [&](int i) {
    int absval = std::abs(d2[i - 1] - d2[i]);
    if (d2[i - 1] * d2[i] < 0 && absval > maxVal) {
      imax = i;
      maxVal = absval;
    }
  };
  if (n > 2 * maxBoxSize) {
    int iforward = n / 2 + 1;
    for (int i = n / 2; i >= 2 && iforward < n - 1; --i, ++iforward) {
      test(i);
      test(iforward);
    }
  } else {
    for (int i = 2; i < n - 1; ++i) test(i);
  }
  if (maxVal == -1 || maxVal < kMinInflectionMag) return -1;
  return imax;
}

// BRMeshRefine::maxloc (BRMeshRefine.cpp:955-967): first index of the largest value.
int maxloc(const int v[3]) {
  int imax = 0;
  for (int i = 1; i < 3; ++i)
    if (v[i] > v[imax]) imax = i;
  return imax;
}

// BRMeshRefine::splitBox (BRMeshRefine.cpp:582-627): halve along the
// longest side until no side exceeds maxBoxSize.
void splitBox(std::vector<Box>& out, Box b, int maxBoxSize) {
  int dir;
  if (longside(b, dir) > maxBoxSize) {
    const int len = (b.lo[dir] + b.hi[dir] + 1) / 2;
    Box hi = b;
    hi.lo[dir] = len;
    b.hi[dir] = len - 1;
    splitBox(out, b, maxBoxSize);
    splitBox(out, hi, maxBoxSize);
  } else {
    out.push_back(b);
  }
}

Box minBoxOf(const IV* begin, const IV* end) {
  Box r(*begin, *begin);
  for (const IV* p = begin + 1; p != end; ++p)
    for (int d = 0; d < 3; ++d) {
      r.lo[d] = std::min(r.lo[d], (*p)[d]);
      r.hi[d] = std::max(r.hi[d], (*p)[d]);
    }
  return r;
}

template <class F>
void parallelFor(size_t n, F fn) {
  hostParallel(n, [&](size_t i) { fn(i); });
}

// Coarse cells of cdom that contain a member of s.  Planes of coarse cells
// are independent (each takes r fine planes), so they run on host threads;
// rows of fine cells are skipped eight bytes at a time while they are empty.
CellSet coarsenSet(const CellSet& s, int r, const Box& cdom) {
  CellSet c(cdom, false);
  const Box& d = s.dom;
  if (d.empty() || cdom.empty()) return c;
  const int kc0 = floordiv(d.lo[2], r), kc1 = floordiv(d.hi[2], r);
  const int nx = d.size(0);
  parallelFor((size_t)(kc1 - kc0 + 1), [&](size_t t) {
    const int kc = kc0 + (int)t;
    for (int k = std::max(d.lo[2], kc * r); k <= std::min(d.hi[2], kc * r + r - 1); ++k)
      for (int j = d.lo[1]; j <= d.hi[1]; ++j) {
        const uint8_t* row = &s.bits[s.at(IV(d.lo[0], j, k))];
        int i = 0;
        while (i < nx) {
          if (i + 8 <= nx) {
            uint64_t w;
            std::memcpy(&w, row + i, 8);
            if (w == 0) {
              i += 8;
              continue;
            }
          }
          if (row[i]) {
            IV q(floordiv(d.lo[0] + i, r), floordiv(j, r), kc);
            if (cdom.contains(q)) c.bits[c.at(q)] = 1;
          }
          ++i;
        }
      }
  });
  return c;
}

CellSet refineSet(const CellSet& s, int r, const Box& fdom) {
  CellSet f(fdom, false);
  const Box& d = s.dom;
  for (int k = d.lo[2]; k <= d.hi[2]; ++k)
    for (int j = d.lo[1]; j <= d.hi[1]; ++j)
      for (int i = d.lo[0]; i <= d.hi[0]; ++i)
        if (s.bits[s.at(IV(i, j, k))]) f.set(Box(IV(i, j, k), IV(i, j, k)).refine(r), true);
  return f;
}

}  // namespace

void NestingSet::build(const CellSet& s) {
  dom = s.dom;
  const int nx = dom.size(0), ny = dom.size(1), nz = dom.size(2);
  sum.assign((size_t)(nx + 1) * (ny + 1) * (nz + 1), 0);
  auto at = [&](int i, int j, int k) { return (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)(ny + 1) * k); };
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        int64_t v = s.bits[s.at(IV(dom.lo[0] + i - 1, dom.lo[1] + j - 1, dom.lo[2] + k - 1))];
        sum[at(i, j, k)] = v + sum[at(i - 1, j, k)] + sum[at(i, j - 1, k)] + sum[at(i, j, k - 1)] -
                           sum[at(i - 1, j - 1, k)] - sum[at(i - 1, j, k - 1)] - sum[at(i, j - 1, k - 1)] +
                           sum[at(i - 1, j - 1, k - 1)];
      }
}

bool NestingSet::containsBox(const Box& b) const {
  if (b.empty()) return true;
  if (!dom.contains(b)) return false;
  const int nx = dom.size(0), ny = dom.size(1);
  auto at = [&](int i, int j, int k) { return (size_t)i + (size_t)(nx + 1) * ((size_t)j + (size_t)(ny + 1) * k); };
  const int i0 = b.lo[0] - dom.lo[0], i1 = b.hi[0] - dom.lo[0] + 1;
  const int j0 = b.lo[1] - dom.lo[1], j1 = b.hi[1] - dom.lo[1] + 1;
  const int k0 = b.lo[2] - dom.lo[2], k1 = b.hi[2] - dom.lo[2] + 1;
  int64_t n = sum[at(i1, j1, k1)] - sum[at(i0, j1, k1)] - sum[at(i1, j0, k1)] - sum[at(i1, j1, k0)] +
              sum[at(i0, j0, k1)] + sum[at(i0, j1, k0)] + sum[at(i1, j0, k0)] - sum[at(i0, j0, k0)];
  return n == b.numPts();
}

MeshRefiner::MeshRefiner(const Box& baseDomain, const std::vector<int>& refRatios, double fillRatio,
                         int blockFactor, int bufferSize, int maxSize)
    : nRef_(refRatios), fillRatio_(fillRatio), blockFactor_(blockFactor), bufferSize_(bufferSize), maxSize_(maxSize) {
  if (blockFactor < 1 || bufferSize < 0 || (maxSize != 0 && blockFactor > maxSize))
    throw std::invalid_argument("cmg: invalid mesh refinement parameters");
  domains_.resize(refRatios.size() + 1);
  domains_[0] = baseDomain;
  for (size_t l = 0; l < refRatios.size(); ++l) domains_[l + 1] = domains_[l].refine(refRatios[l]);
  // MeshRefine::computeLocalBlockFactors (MeshRefine.cpp:776-795)
  blockFactors_.resize(refRatios.size());
  for (size_t l = 0; l < refRatios.size(); ++l) {
    blockFactors_[l] = (blockFactor + refRatios[l] - 1) / refRatios[l];
    if (!isPow2(blockFactors_[l])) throw std::invalid_argument("cmg: ceil(blockFactor/nRef) must be a power of 2");
  }
}

void MeshRefiner::makeBoxes(std::vector<Box>& mesh, std::vector<IV>& tags, const NestingSet& pnd, const Box& domain,
                            int maxBoxSize, int totalBufferSize) const {
  mesh.clear();
  if (tags.empty()) return;
  makeBoxesRec(mesh, tags.data(), tags.data() + tags.size(), pnd, domain, maxBoxSize, totalBufferSize);
}

void MeshRefiner::makeBoxesRec(std::vector<Box>& mesh, IV* begin, IV* end, const NestingSet& pnd,
                               const Box& domain, int maxBoxSize, int totalBufferSize) const {
  const int64_t ntags = end - begin;
  if (ntags == 0) return;
  const Box minbox = minBoxOf(begin, end);
  // MeshRefine::properlyNested, PND mode 1 (MeshRefine.cpp:998-1050)
  const bool nested = pnd.containsBox(minbox.grow(totalBufferSize) & domain);
  if (!nested && ntags == 1) return;
  if ((double)ntags >= (double)minbox.numPts() * fillRatio_ && nested) {
    if (maxBoxSize > 0)
      splitBox(mesh, minbox, maxBoxSize);
    else
      mesh.push_back(minbox);
    return;
  }
  // BRMeshRefine::splitTagsInBestDimension (BRMeshRefine.cpp:464-552)
  std::vector<int> traces[3];
  for (int d = 0; d < 3; ++d) traces[d].assign(minbox.size(d), 0);
  for (IV* p = begin; p != end; ++p)
    for (int d = 0; d < 3; ++d) traces[d][(*p)[d] - minbox.lo[d]]++;
  int hole[3], infl[3];
  for (int d = 0; d < 3; ++d) {
    hole[d] = findSplit(traces[d], maxBoxSize);
    infl[d] = findInflection(traces[d], maxBoxSize);
  }
  const int bh = maxloc(hole), bi = maxloc(infl);
  int dim, index;
  if (hole[bh] >= 0) {
    dim = bh;
    index = hole[bh] + minbox.lo[bh];
  } else if (infl[bi] >= 0) {
    dim = bi;
    index = infl[bi] + minbox.lo[bi];
  } else {
    longside(minbox, dim);
    index = (minbox.lo[dim] + minbox.hi[dim] + 1) / 2;
  }
  IV* mid = std::partition(begin, end, [&](const IV& p) { return p[dim] < index; });
  makeBoxesRec(mesh, begin, mid, pnd, domain, maxBoxSize, totalBufferSize);
  makeBoxesRec(mesh, mid, end, pnd, domain, maxBoxSize, totalBufferSize);
}

int MeshRefiner::regrid(std::vector<std::vector<Box>>& newMeshes, std::vector<CellSet>& tags, int baseLevel,
                        int topLevel, const std::vector<std::vector<Box>>& oldMeshes) const {
  int level = std::min(topLevel, (int)tags.size() - 1);
  for (; level >= baseLevel; --level)
    if (!tags[level].empty()) break;
  if (level < baseLevel) {
    newMeshes.assign(oldMeshes.begin(), oldMeshes.end());
    return baseLevel;
  }
  const int top = level;
  newMeshes.assign(top + 2, std::vector<Box>());
  if (!domains_[baseLevel].coarsenable(blockFactor_))
    throw std::invalid_argument("cmg: domain and blocking factor incompatible");
  // Blocked tags, domains and buffers per level.
  std::vector<Box> dom(top + 1);
  std::vector<int> blockedBuffer(top + 1), totalBuffer(top + 1, 0);
  std::vector<CellSet> btags(top + 1);
  for (int l = baseLevel; l <= top; ++l) {
    dom[l] = domains_[l].coarsen(blockFactors_[l]);
    tags[l].intersect(domains_[l]);
    btags[l] = coarsenSet(tags[l], blockFactors_[l], dom[l]);
    blockedBuffer[l] = (bufferSize_ + blockFactors_[l] - 1) / blockFactors_[l];
  }
  // MeshRefine::makePNDs (MeshRefine.cpp:924-996), mode 1.
  std::vector<CellSet> pnds(top + 1);
  pnds[baseLevel].define(dom[baseLevel], false);
  for (const Box& b : oldMeshes[baseLevel]) pnds[baseLevel].set(b.coarsen(blockFactors_[baseLevel]), true);
  for (int l = baseLevel; l <= top; ++l) {
    totalBuffer[l] += blockedBuffer[l];
    if (top - l > 0) {
      const int allInOne = blockFactors_[l] * nRef_[l] / blockFactors_[l + 1];
      totalBuffer[l + 1] = totalBuffer[l] * allInOne;
      pnds[l + 1] = refineSet(pnds[l], allInOne, dom[l + 1]);
    }
  }
  for (int l = baseLevel; l <= top; ++l)
    for (size_t q = 0; q < btags[l].bits.size(); ++q) btags[l].bits[q] &= pnds[l].bits[q];
  // New meshes from the top level down, each level's tags unioned with the
  // buffered boxes of the level above.
  std::vector<Box> lvlboxes;
  for (int l = top; l >= baseLevel; --l) {
    for (const Box& b : lvlboxes) btags[l].set(b, true);  // buildSupport
    const int maxBoxSizeLevel = maxSize_ / (blockFactors_[l] * nRef_[l]);
    std::vector<IV> cells;
    const Box& d = btags[l].dom;
    for (int k = d.lo[2]; k <= d.hi[2]; ++k)
      for (int j = d.lo[1]; j <= d.hi[1]; ++j)
        for (int i = d.lo[0]; i <= d.hi[0]; ++i)
          if (btags[l].bits[btags[l].at(IV(i, j, k))]) cells.push_back(IV(i, j, k));
    NestingSet pnd;
    pnd.build(pnds[l]);
    makeBoxes(lvlboxes, cells, pnd, dom[l], maxBoxSizeLevel, totalBuffer[l]);
    newMeshes[l + 1] = lvlboxes;
    for (Box& b : newMeshes[l + 1]) b = b.refine(blockFactors_[l] * nRef_[l]);
    if (l > baseLevel) {
      const int allInOne = blockFactors_[l - 1] * nRef_[l - 1] / blockFactors_[l];
      for (Box& b : lvlboxes) b = (b.grow(blockedBuffer[l]) & dom[l]).coarsen(allInOne);
    }
  }
  for (int i = 0; i <= baseLevel; ++i) newMeshes[i] = oldMeshes[i];
  int finest = top + 1;
  while (finest > baseLevel && newMeshes[finest].empty()) --finest;
  return finest;
}

namespace {


// Tags of one level, grown by one cell and clipped to the level's domain:
// cells of `grids` with |rhs| > thresh * max|rhs| (oracle/driver.cpp, after
// VClocalFuncs.cpp:586-624 with a strict comparison).
CellSet levelTags(const std::vector<Box>& grids, const Box& domain, double dx, const cmg_synth::Bumps& bumps,
                  double thresh) {
  std::vector<std::vector<double>> vals(grids.size());
  std::vector<double> boxMax(grids.size(), 0.0);
  parallelFor(grids.size(), [&](size_t b) {
    const Box& bx = grids[b];
    vals[b].resize(bx.numPts());
    size_t q = 0;
    double m = 0.0;
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
      for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
        for (int i = bx.lo[0]; i <= bx.hi[0]; ++i) {
          double v = bumps.eval((i + 0.5) * dx, (j + 0.5) * dx, (k + 0.5) * dx);
          vals[b][q++] = v;
          m = std::max(m, std::fabs(v));
        }
    boxMax[b] = m;
  });
  double maxRHS = 0.0;
  for (double m : boxMax) maxRHS = std::max(maxRHS, m);
  const double tagVal = maxRHS * thresh;
  CellSet tags(domain, false);
  for (size_t b = 0; b < grids.size(); ++b) {
    const Box& bx = grids[b];
    size_t q = 0;
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
      for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
        for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
          if (std::fabs(vals[b][q++]) > tagVal) tags.set(Box(IV(i, j, k), IV(i, j, k)).grow(1), true);
  }
  return tags;
}

}  // namespace

std::vector<std::vector<Box>> syntheticHierarchy(int n0, int numLevels, int maxBox, int blockFactor, double fillRatio,
                                                 uint64_t seed, double thresh, LevelTagger* tagger) {
  if (n0 < 1 || numLevels < 1) throw std::invalid_argument("cmg: invalid hierarchy parameters");
  cmg_synth::Problem prob(seed);
  std::vector<Box> domains(numLevels);
  std::vector<double> dxs(numLevels);
  domains[0] = Box(IV(0, 0, 0), IV(n0 - 1, n0 - 1, n0 - 1));
  dxs[0] = 1.0 / n0;
  for (int l = 1; l < numLevels; ++l) {
    domains[l] = domains[l - 1].refine(2);
    dxs[l] = dxs[l - 1] / 2;
  }
  std::vector<std::vector<Box>> grids(numLevels), oldBoxes(numLevels), newBoxes;
  oldBoxes[0] = domainSplit(domains[0], maxBox, blockFactor);
  grids[0] = Layout(oldBoxes[0]).boxes;
  int topLevel = 0;
  if (numLevels > 1) {
    MeshRefiner refiner(domains[0], std::vector<int>(std::max(numLevels, 2), 2), fillRatio, blockFactor, 2, maxBox);
    bool more = true;
    std::vector<CellSet> cached(numLevels);
    std::vector<std::vector<Box>> cachedGrids(numLevels);
    std::vector<char> haveCache(numLevels, 0);
    while (more) {
      more = false;
      const int oldTop = topLevel;
      for (int l = 0; l <= topLevel; ++l) {
        if (!haveCache[l] || !(cachedGrids[l] == grids[l])) {
          if (tagger)
            tagger->tags(grids[l], domains[l], dxs[l], prob.bumps, thresh, cached[l]);
          else
            cached[l] = levelTags(grids[l], domains[l], dxs[l], prob.bumps, thresh);
          cachedGrids[l] = grids[l];
          haveCache[l] = 1;
        }
      }
      // regrid reads levels 0..topLevel and only clips each tag set to its
      // level's domain, which these sets already are: the cache is passed
      // as it is.
      int newFinest = refiner.regrid(newBoxes, cached, 0, topLevel, oldBoxes);
      if (newFinest > topLevel) topLevel++;
      oldBoxes = newBoxes;
      oldBoxes.resize(std::max<size_t>(oldBoxes.size(), numLevels));
      for (int l = 1; l <= topLevel; ++l) grids[l] = Layout(l < (int)newBoxes.size() ? newBoxes[l] : std::vector<Box>()).boxes;
      if (topLevel < numLevels - 1 && topLevel > oldTop) more = true;
    }
  }
  grids.resize(topLevel + 1);
  return grids;
}

}  // namespace cmg
