// ORACLE — test infrastructure only.  Never linked into the product.
//
// The seeded synthetic hierarchies of the benchmark workloads built with the
// reference's own grid generation and data types, shared by the oracle
// driver (driver.cpp) and the drop-in check (dropin.cpp).
//
// Grid generation follows the reference example drivers:
//   base level   releasedExamples/AMRPoisson/execCell/poissonSolve.cpp:296-317
//                (domainSplit + LoadBalance + DisjointBoxLayout)
//   finer levels releasedExamples/AMRPoisson/execVariableCoefficient/
//                VClocalFuncs.cpp:398-480 (tag |rhs| vs thresh*max|rhs|,
//                grow tags by 1, BRMeshRefine with nesting radius 2, one new
//                level per pass)
#ifndef CMG_ORACLE_PROBLEM_H
#define CMG_ORACLE_PROBLEM_H

#include <chrono>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "AMRMultiGrid.H"
#include "BCFunc.H"
#include "BRMeshRefine.H"
#include "BoxIterator.H"
#include "DisjointBoxLayout.H"
#include "FArrayBox.H"
#include "FluxBox.H"
#include "LevelData.H"
#include "LoadBalance.H"
#include "ProblemDomain.H"
#include "REAL.H"
#include "synthetic.H"

typedef LevelData<FArrayBox> LDF;

// Homogeneous Dirichlet on domain faces, first order (ghost = -interior), as
// the reference driver's ParseBC (execCell/poissonSolve.cpp:76-119).
static void zeroValue(Real*, int*, Side::LoHiSide*, Real* a_values) { a_values[0] = 0.; }

// Homogeneous boundary type of each domain face (x-lo, x-hi, y-lo, y-hi,
// z-lo, z-hi): 0 Dirichlet (the examples' ParseBC), 1 Neumann (walls and
// inflow in the AMRINS projection's pressure BC function,
// releasedExamples/AMRINS/BCutil/PhysBCUtil.cpp:427-473), 2 periodic (the
// direction's ProblemDomain periodicity; both faces of a direction).  Set
// from the bc=<six letters D/N/P> argument.
static int g_faceBC[6] = {0, 0, 0, 0, 0, 0};
static void setFaceBC(const std::string& a_s) {
  for (int f = 0; f < 6; ++f) {
    const char c = f < (int)a_s.size() ? a_s[f] : 'D';
    g_faceBC[f] = c == 'N' ? 1 : c == 'P' ? 2 : 0;
  }
}
static std::string faceBCString() {
  std::string s;
  for (int f = 0; f < 6; ++f) s += g_faceBC[f] == 1 ? 'N' : g_faceBC[f] == 2 ? 'P' : 'D';
  return s;
}

static void domainBC(FArrayBox& a_state, const Box& a_valid, const ProblemDomain& a_domain,
                     Real a_dx, bool a_homogeneous) {
  if (!a_domain.domainBox().contains(a_state.box())) {
    for (int i = 0; i < CH_SPACEDIM; ++i) {
      if (!a_domain.isPeriodic(i)) {
        for (SideIterator sit; sit.ok(); ++sit) {
          Box g = adjCellBox(a_valid, i, sit(), 1);
          if (a_domain.domainBox().contains(g)) continue;
          if (g_faceBC[2 * i + (sit() == Side::Hi ? 1 : 0)])
            NeumBC(a_state, a_valid, a_dx, true, zeroValue, i, sit());
          else
            DiriBC(a_state, a_valid, a_dx, true, zeroValue, i, sit(), 1);
        }
      }
    }
  }
}

// Records max-norm of the composite residual at the start of every iteration.
class ResidualRecorder : public AMRMultiGridInspector<LDF> {
 public:
  std::vector<double> norms;
  std::vector<double> stamps;  // wall time at the start of each iteration
  void recordResiduals(const Vector<LDF*>& r, int lmin, int lmax, int) override {
    stamps.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count());
    double m = 0;
    for (int l = lmin; l <= lmax; ++l)
      for (DataIterator dit = r[l]->dataIterator(); dit.ok(); ++dit)
        m = std::max(m, (*r[l])[dit].norm(r[l]->box(dit()), 0, 0, 1));
    norms.push_back(m);
  }
  void recordCorrections(const Vector<LDF*>&, int, int, int) override {}
};

static void fillRHS(LDF& rhs, Real dx, const cmg_synth::Bumps& bumps) {
  for (DataIterator dit = rhs.dataIterator(); dit.ok(); ++dit) {
    FArrayBox& f = rhs[dit];
    const Box& b = rhs.box(dit());
    for (BoxIterator bit(b); bit.ok(); ++bit) {
      IntVect iv = bit();
      f(iv, 0) = bumps.eval((iv[0] + 0.5) * dx, (iv[1] + 0.5) * dx, (iv[2] + 0.5) * dx);
    }
  }
}

struct OracleProblem {
  // inputs
  int n0 = 64, numLevels = 1, maxBox = 32, blockFactor = 8, opType = 0;
  Real fillRatio = 0.75, alpha = 0.0, beta = 1.0, thresh = 0.1;
  unsigned long long seed = 20261203ULL;
  std::string boxfile;
  // outputs
  Vector<ProblemDomain> domains;
  Vector<Real> dxs;
  Vector<DisjointBoxLayout> grids;
  int finest = 0, nlev = 1;
  Vector<LDF*> phi, rhs;
  Vector<RefCountedPtr<LDF> > aCoef;
  Vector<RefCountedPtr<LevelData<FluxBox> > > bCoef;
};

// Builds grids and data; returns 0, or 2 on a bad box file.
inline int buildProblem(OracleProblem& P) {
  const int n0 = P.n0, numLevels = P.numLevels, maxBox = P.maxBox, blockFactor = P.blockFactor, opType = P.opType;
  const Real fillRatio = P.fillRatio, thresh = P.thresh;
  const std::string& boxfile = P.boxfile;
  cmg_synth::Problem prob(P.seed);

  // Domains and dx per level (ratio 2).
  Vector<int> refRatios(std::max(numLevels, 2), 2);
  Vector<ProblemDomain> domains(numLevels);
  Vector<Real> dxs(numLevels);
  bool periodic[CH_SPACEDIM] = {g_faceBC[0] == 2, g_faceBC[2] == 2, g_faceBC[4] == 2};
  domains[0] = ProblemDomain(IntVect::Zero, (n0 - 1) * IntVect::Unit, periodic);
  dxs[0] = 1.0 / n0;
  for (int l = 1; l < numLevels; ++l) {
    domains[l] = domains[l - 1];
    domains[l].refine(2);
    dxs[l] = dxs[l - 1] / 2;
  }

  // Base level.
  Vector<DisjointBoxLayout> grids(numLevels);
  Vector<Vector<Box> > oldBoxes(numLevels), newBoxes(numLevels);
  domainSplit(domains[0], oldBoxes[0], maxBox, blockFactor);
  {
    Vector<int> procs(oldBoxes[0].size(), 0);
    LoadBalance(procs, oldBoxes[0]);
    grids[0].define(oldBoxes[0], procs, domains[0]);
  }
  // Finer levels: VClocalFuncs.cpp:398-480, or a given layout (boxfile=:
  // "nlev" then per level "nbox" and nbox lines "lo0 lo1 lo2 hi0 hi1 hi2").
  int topLevel = 0;
  if (!boxfile.empty()) {
    FILE* bf = std::fopen(boxfile.c_str(), "r");
    if (!bf) {
      std::fprintf(stderr, "oracle: cannot open %s\n", boxfile.c_str());
      return 2;
    }
    int nl = 0;
    if (std::fscanf(bf, "%d", &nl) != 1 || nl < 1 || nl > numLevels) return 2;
    for (int l = 0; l < nl; ++l) {
      int nb = 0;
      if (std::fscanf(bf, "%d", &nb) != 1) return 2;
      Vector<Box> bl;
      for (int b = 0; b < nb; ++b) {
        int v[6];
        for (int k = 0; k < 6; ++k)
          if (std::fscanf(bf, "%d", &v[k]) != 1) return 2;
        bl.push_back(Box(IntVect(v[0], v[1], v[2]), IntVect(v[3], v[4], v[5])));
      }
      Vector<int> procs(bl.size(), 0);
      LoadBalance(procs, bl);
      grids[l] = DisjointBoxLayout(bl, procs, domains[l]);
    }
    std::fclose(bf);
    topLevel = nl - 1;
  } else if (numLevels > 1) {
    BRMeshRefine meshrefine(domains[0], refRatios, fillRatio, blockFactor, 2, maxBox);
    bool more = true;
    while (more) {
      more = false;
      int oldTop = topLevel;
      Vector<IntVectSet> tags(topLevel + 1);
      for (int l = 0; l <= topLevel; ++l) {
        LDF rhs(grids[l], 1, IntVect::Zero);
        fillRHS(rhs, dxs[l], prob.bumps);
        Real maxRHS = norm(rhs, rhs.interval(), 0);
        Real tagVal = maxRHS * thresh;
        IntVectSet local;
        for (DataIterator dit = rhs.dataIterator(); dit.ok(); ++dit) {
          const Box b = grids[l].get(dit());
          for (BoxIterator bit(b); bit.ok(); ++bit)
            if (std::fabs(rhs[dit](bit(), 0)) > tagVal) local |= bit();
        }
        local.grow(1);
        local &= domains[l].domainBox();
        tags[l] = local;
      }
      int newFinest = meshrefine.regrid(newBoxes, tags, 0, topLevel, oldBoxes);
      if (newFinest > topLevel) topLevel++;
      oldBoxes = newBoxes;
      for (int l = 1; l <= topLevel; ++l) {
        Vector<int> procs(newBoxes[l].size(), 0);
        LoadBalance(procs, newBoxes[l]);
        grids[l] = DisjointBoxLayout(newBoxes[l], procs, domains[l]);
      }
      if (topLevel < numLevels - 1 && topLevel > oldTop) more = true;
    }
  }
  const int finest = topLevel;
  const int nlev = finest + 1;

  // Data.
  Vector<LDF*> phi(nlev, NULL), rhs(nlev, NULL);
  Vector<RefCountedPtr<LDF> > aCoef(nlev);
  Vector<RefCountedPtr<LevelData<FluxBox> > > bCoef(nlev);
  for (int l = 0; l < nlev; ++l) {
    phi[l] = new LDF(grids[l], 1, IntVect::Unit);
    rhs[l] = new LDF(grids[l], 1, IntVect::Zero);
    fillRHS(*rhs[l], dxs[l], prob.bumps);
    if (opType == 1) {
      aCoef[l] = RefCountedPtr<LDF>(new LDF(grids[l], 1, IntVect::Zero));
      bCoef[l] = RefCountedPtr<LevelData<FluxBox> >(new LevelData<FluxBox>(grids[l], 1, IntVect::Zero));
      Real dx = dxs[l];
      for (DataIterator dit = grids[l].dataIterator(); dit.ok(); ++dit) {
        FArrayBox& a = (*aCoef[l])[dit];
        for (BoxIterator bit(a.box()); bit.ok(); ++bit) {
          IntVect iv = bit();
          a(iv, 0) = prob.acoef.eval((iv[0] + 0.5) * dx, (iv[1] + 0.5) * dx, (iv[2] + 0.5) * dx);
        }
        for (int d = 0; d < 3; ++d) {
          FArrayBox& b = (*bCoef[l])[dit][d];
          for (BoxIterator bit(b.box()); bit.ok(); ++bit) {
            IntVect iv = bit();
            double x[3];
            for (int e = 0; e < 3; ++e) x[e] = (e == d) ? iv[e] * dx : (iv[e] + 0.5) * dx;
            b(iv, 0) = prob.bcoef.eval(x[0], x[1], x[2]);
          }
        }
      }
    }
  }

  P.domains = domains;
  P.dxs = dxs;
  P.grids = grids;
  P.finest = finest;
  P.nlev = nlev;
  P.phi = phi;
  P.rhs = rhs;
  P.aCoef = aCoef;
  P.bCoef = bCoef;
  return 0;
}

#endif
