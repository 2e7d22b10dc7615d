// ORACLE — test infrastructure only.  Never linked into the product.
//
// Runs the reference's heat solvers for a few steps on the seeded synthetic
// hierarchies (problem.H): BackwardEuler (lib/src/AMRElliptic/
// BackwardEuler.cpp: oneStep, createEulerRHS, solveHelm with
// setAlphaAndBeta(1, -dt) on every operator, then AMRMultiGrid::solve from
// the old solution) or, with scheme=tga, AMRTGA (AMRTGA.H:420-560: two
// Helmholtz solves per step).  The initial state and the source are both the
// seeded right-hand side.  Dumps the exit status and V-cycle count of every
// solve (for TGA the exit status after each step's second solve) and the
// final phi on every level.
//
// Usage: cmg_oracle_heat key=value ... out=<prefix>
//   n0 levels maxbox block fill op alpha beta seed thresh (as cmg_oracle)
//   pre post bottom iters eps hang dt=1e-3 steps=3 scheme=euler|tga
// Writes <prefix>.json and <prefix>.bin (per level, per box in layout order,
// valid cells x-fastest: phi after the last step).

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "AMRMultiGrid.H"
#include "AMRPoissonOp.H"
#include "BCFunc.H"
#include "AMRTGA.H"
#include "BackwardEuler.H"
#include "BiCGStabSolver.H"
#include "VCAMRPoissonOp2.H"
#include "problem.H"

static std::map<std::string, std::string> g_args;
static double argd(const char* k, double d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? d : std::atof(it->second.c_str());
}
static int argi(const char* k, int d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? d : std::atoi(it->second.c_str());
}

// The iteration index of every residual report: a new solve starts at 0.
class IterRecorder : public AMRMultiGridInspector<LDF> {
 public:
  std::vector<int> iters;
  void recordResiduals(const Vector<LDF*>&, int, int, int iter) override { iters.push_back(iter); }
  void recordCorrections(const Vector<LDF*>&, int, int, int) override {}
};

int main(int argc, char** argv) {
  for (int a = 1; a < argc; ++a) {
    const char* eq = std::strchr(argv[a], '=');
    if (eq) g_args[std::string(argv[a], eq - argv[a])] = std::string(eq + 1);
  }
  if (g_args.count("bc")) setFaceBC(g_args["bc"]);
  OracleProblem P;
  P.n0 = argi("n0", 32);
  P.numLevels = argi("levels", 1);
  P.maxBox = argi("maxbox", 32);
  P.blockFactor = argi("block", 8);
  P.fillRatio = argd("fill", 0.75);
  P.opType = argi("op", 0);
  P.alpha = argd("alpha", 1.0);
  P.beta = argd("beta", 1.0);
  P.seed = (unsigned long long)argd("seed", 20261203.0);
  P.thresh = argd("thresh", 0.1);
  const int pre = argi("pre", 4), post = argi("post", 4), bottom = argi("bottom", 4), iters = argi("iters", 100);
  const Real eps = argd("eps", 1e-10), hang = argd("hang", 1e-10), dt = argd("dt", 1e-3);
  const int steps = argi("steps", 3);
  const bool tga = g_args.count("scheme") && g_args["scheme"] == "tga";
  const std::string out = g_args.count("out") ? g_args["out"] : std::string("heat_out");
  if (buildProblem(P) != 0) return 2;
  const int nlev = P.nlev, lmax = P.finest;

  Vector<int> rr(nlev, 2);
  AMRLevelOpFactory<LDF>* factory = NULL;
  if (P.opType == 0) {
    AMRPoissonOpFactory* f = new AMRPoissonOpFactory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    factory = f;
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    factory = f;
  }
  BiCGStabSolver<LDF> bottomSolver;
  bottomSolver.m_verbosity = 0;
  RefCountedPtr<AMRMultiGrid<LDF> > solver(new AMRMultiGrid<LDF>());
  solver->define(P.domains[0], *factory, &bottomSolver, nlev);
  solver->setSolverParameters(pre, post, bottom, 1, iters, eps, hang, 1e-30);
  solver->m_verbosity = 0;
  RefCountedPtr<AMRMultiGridInspector<LDF> > insp(new ResidualRecorder);
  solver->addInspector(insp);
  ResidualRecorder* rec = static_cast<ResidualRecorder*>(&(*insp));

  // phiOld = the seeded right-hand side (valid cells), source = the same,
  // with one ghost layer (TGA applies the operator to the source).
  Vector<LDF*> phiOld(nlev), phiNew(nlev), src(nlev);
  for (int l = 0; l < nlev; ++l) {
    phiOld[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    phiNew[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    src[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) {
      (*phiOld[l])[dit()].setVal(0.0);
      (*phiNew[l])[dit()].setVal(0.0);
      (*src[l])[dit()].setVal(0.0);
      (*phiOld[l])[dit()].copy((*P.rhs[l])[dit()], P.grids[l][dit()]);
      (*src[l])[dit()].copy((*P.rhs[l])[dit()], P.grids[l][dit()]);
    }
  }
  std::vector<int> exits, vcycles;
  if (!tga) {
    BackwardEuler be(solver, *factory, P.domains[0], rr, nlev, 0);
    for (int n = 0; n < steps; ++n) {
      const size_t before = rec->norms.size();
      be.oneStep(phiNew, phiOld, src, dt, 0, lmax, false);
      exits.push_back(solver->m_exitStatus);
      vcycles.push_back((int)(rec->norms.size() - before));
      std::swap(phiOld, phiNew);
    }
  } else {
    RefCountedPtr<AMRMultiGridInspector<LDF> > itInsp(new IterRecorder);
    solver->addInspector(itInsp);
    IterRecorder* its = static_cast<IterRecorder*>(&(*itInsp));
    // AMRTGA calls solveNoInit: the set-up AMRMultiGrid::solve would do first.
    solver->init(phiNew, src, lmax, 0);
    solver->setBottomSolver(lmax, 0);
    AMRTGA<LDF> tgaSolver(solver, *factory, P.domains[0], rr, nlev, 0);
    for (int n = 0; n < steps; ++n) {
      const size_t before = its->iters.size();
      tgaSolver.oneStep(phiNew, phiOld, src, dt, 0, lmax, 0.0);
      exits.push_back(solver->m_exitStatus);
      // split this step's reports into its two solves
      std::vector<int> counts;
      for (size_t k = before; k < its->iters.size(); ++k) {
        if (its->iters[k] == 0) counts.push_back(0);
        counts.back()++;
      }
      if (counts.size() != 2) return 3;
      vcycles.push_back(counts[0]);
      vcycles.push_back(counts[1]);
      std::swap(phiOld, phiNew);
    }
  }

  FILE* js = std::fopen((out + ".json").c_str(), "w");
  std::fprintf(js, "{\"dt\": %.17g, \"steps\": %d, \"scheme\": \"%s\", \"exit_status\": [", dt, steps,
               tga ? "tga" : "euler");
  for (size_t n = 0; n < exits.size(); ++n) std::fprintf(js, "%s%d", n ? "," : "", exits[n]);
  std::fprintf(js, "], \"iterations\": [");
  for (size_t n = 0; n < vcycles.size(); ++n) std::fprintf(js, "%s%d", n ? "," : "", vcycles[n]);
  std::fprintf(js, "]}\n");
  std::fclose(js);
  FILE* bin = std::fopen((out + ".bin").c_str(), "wb");
  for (int l = 0; l < nlev; ++l)
    for (LayoutIterator lit = P.grids[l].layoutIterator(); lit.ok(); ++lit) {
      const Box& b = P.grids[l][lit];
      const FArrayBox& fab = (*phiOld[l])[DataIndex(lit())];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
          for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) {
            double v = fab(IntVect(i, j, k), 0);
            std::fwrite(&v, sizeof(double), 1, bin);
          }
    }
  std::fclose(bin);
  std::printf("heat: levels=%d steps=%d exits=%d..%d vcycles=%d..%d\n", nlev, steps, exits.front(), exits.back(),
              vcycles.front(), vcycles.back());
  return 0;
}
