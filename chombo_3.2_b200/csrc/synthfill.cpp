#include "synthfill.H"

#include <algorithm>
#include <thread>
#include <vector>

#include "hostpool.H"
#include "synthetic.H"

namespace cmg {

namespace {

template <class F>
void parallelBoxes(size_t nbox, F fn) {
  hostParallel(nbox, [&](size_t b) { fn(b); });
}

}  // namespace

void fillSynthetic(Solver& S, bool vc, uint64_t seed) {
  cmg_synth::Problem prob(seed);
  for (int l = 0; l < S.numLevels(); ++l) {
    const LevelPlan& L = S.level(l);
    const double dx = L.dx;
    std::vector<int64_t> off(L.grids.size() + 1, 0);
    for (size_t b = 0; b < L.grids.size(); ++b) off[b + 1] = off[b] + L.grids[b].numPts();
    std::vector<double> rhs(off.back()), a;
    if (vc) a.resize(off.back());
    parallelBoxes(L.grids.size(), [&](size_t b) {
      const Box& B = L.grids[b];
      int64_t q = off[b];
      for (int k = B.lo[2]; k <= B.hi[2]; ++k)
        for (int j = B.lo[1]; j <= B.hi[1]; ++j)
          for (int i = B.lo[0]; i <= B.hi[0]; ++i, ++q) {
            double x = (i + 0.5) * dx, y = (j + 0.5) * dx, z = (k + 0.5) * dx;
            rhs[q] = prob.bumps.eval(x, y, z);
            if (!a.empty()) a[q] = prob.acoef.eval(x, y, z);
          }
    });
    S.setRHS(l, rhs.data(), false);
    if (!vc) continue;
    S.setACoef(l, a.data(), false);
    for (int d = 0; d < 3; ++d) {
      std::vector<int64_t> fo(L.grids.size() + 1, 0);
      for (size_t b = 0; b < L.grids.size(); ++b) {
        Box fb = L.grids[b];
        fb.hi[d] += 1;
        fo[b + 1] = fo[b] + fb.numPts();
      }
      std::vector<double> bc(fo.back());
      parallelBoxes(L.grids.size(), [&](size_t b) {
        Box fb = L.grids[b];
        fb.hi[d] += 1;
        int64_t q = fo[b];
        for (int k = fb.lo[2]; k <= fb.hi[2]; ++k)
          for (int j = fb.lo[1]; j <= fb.hi[1]; ++j)
            for (int i = fb.lo[0]; i <= fb.hi[0]; ++i, ++q) {
              int iv[3] = {i, j, k};
              double x[3];
              for (int e = 0; e < 3; ++e) x[e] = (e == d) ? iv[e] * dx : (iv[e] + 0.5) * dx;
              bc[q] = prob.bcoef.eval(x[0], x[1], x[2]);
            }
      });
      S.setBCoef(l, d, bc.data(), false);
    }
  }
  if (vc) S.finalizeCoefficients();
}

}  // namespace cmg
