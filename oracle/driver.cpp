// ORACLE — test infrastructure only.  Never linked into the product.
//
// Drives the reference's own AMRMultiGrid::solve (lib/src/AMRElliptic/
// AMRMultiGrid.H:894-1124) over AMRPoissonOp or VCAMRPoissonOp2 on the seeded
// synthetic hierarchies of the benchmark workloads, and dumps every artefact
// the GPU path is checked against: box layouts, exchange/copyTo motion plans,
// the per-iteration residual norms, the exit status and phi on every level.
//
// Grid generation follows the reference example drivers:
//   base level   releasedExamples/AMRPoisson/execCell/poissonSolve.cpp:296-317
//                (domainSplit + LoadBalance + DisjointBoxLayout)
//   finer levels releasedExamples/AMRPoisson/execVariableCoefficient/
//                VClocalFuncs.cpp:398-480 (tag |rhs| vs thresh*max|rhs|,
//                grow tags by 1, BRMeshRefine with nesting radius 2, one new
//                level per pass)
// Solver set-up follows poissonSolve.cpp:533-583 and VClocalFuncs.cpp:528-556.
//
// Usage: cmg_oracle key=value ... out=<prefix>
//   n0=64 levels=1 maxbox=32 block=8 fill=0.75 op=0|1 alpha=0 beta=1
//   seed=20261203 thresh=0.1 pre=4 post=4 bottom=4 iters=100 eps=1e-10
//   hang=1e-10 dumpphi=1 plansonly=0 (1: write <prefix>.plans and stop)
// Writes <prefix>.json (metadata, boxes, plans, residual history) and
// <prefix>.bin (raw little-endian doubles: per level, per box in layout
// order, valid cells x-fastest: rhs, phi, then for op=1 acoef and the three
// face coefficient arrays over their face boxes).

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <map>
#include <vector>
#include <random>
#include <chrono>

#include "REAL.H"
#include "Box.H"
#include "ProblemDomain.H"
#include "DisjointBoxLayout.H"
#include "LevelData.H"
#include "FArrayBox.H"
#include "FluxBox.H"
#include "BRMeshRefine.H"
#include "LoadBalance.H"
#include "BoxIterator.H"
#include "AMRMultiGrid.H"
#include "AMRPoissonOp.H"
#include "VCAMRPoissonOp2.H"
#include "BiCGStabSolver.H"
#include "BCFunc.H"
#include "Copier.H"
#include "CH_Timer.H"
#include "parstream.H"

#include "problem.H"
#include "synthetic.H"

static std::map<std::string, std::string> g_args;

static double argd(const char* k, double d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? d : std::atof(it->second.c_str());
}
static int argi(const char* k, int d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? d : std::atoi(it->second.c_str());
}
static std::string args(const char* k, const char* d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? std::string(d) : it->second;
}

static void writeBox(FILE* f, const Box& b) {
  std::fprintf(f, "[%d,%d,%d,%d,%d,%d]", b.smallEnd(0), b.smallEnd(1), b.smallEnd(2),
               b.bigEnd(0), b.bigEnd(1), b.bigEnd(2));
}

static void writeCopier(FILE* f, const Copier& c) {
  std::fprintf(f, "[");
  bool first = true;
  for (CopyIterator it(c, CopyIterator::LOCAL); it.ok(); ++it) {
    const MotionItem& m = it();
    std::fprintf(f, "%s[%d,%d,", first ? "" : ",", m.fromIndex.intCode(), m.toIndex.intCode());
    writeBox(f, m.fromRegion);
    std::fprintf(f, ",");
    writeBox(f, m.toRegion);
    std::fprintf(f, "]");
    first = false;
  }
  std::fprintf(f, "]");
}

static void writeFab(FILE* bin, const FArrayBox& fab, const Box& b) {
  for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
    for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
      for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) {
        double v = fab(IntVect(i, j, k), 0);
        std::fwrite(&v, sizeof(double), 1, bin);
      }
}

int main(int argc, char** argv) {
  for (int a = 1; a < argc; ++a) {
    const char* eq = std::strchr(argv[a], '=');
    if (!eq) continue;
    g_args[std::string(argv[a], eq - argv[a])] = std::string(eq + 1);
  }
  if (g_args.count("bc")) setFaceBC(g_args["bc"]);
  const int n0 = argi("n0", 64);
  const int numLevels = argi("levels", 1);
  const int maxBox = argi("maxbox", 32);
  const int blockFactor = argi("block", 8);
  const Real fillRatio = argd("fill", 0.75);
  const int opType = argi("op", 0);
  const Real alpha = argd("alpha", 0.0);
  const Real beta = argd("beta", 1.0);
  const unsigned long long seed = (unsigned long long)argd("seed", 20261203.0);
  const Real thresh = argd("thresh", 0.1);
  const int pre = argi("pre", 4), post = argi("post", 4), bottom = argi("bottom", 4);
  const int iterMax = argi("iters", 100);
  const Real eps = argd("eps", 1e-10), hang = argd("hang", 1e-10);
  const int dumpPhi = argi("dumpphi", 1);
  const int repeat = argi("repeat", 1);
  const std::string out = args("out", "oracle_out");

  OracleProblem P;
  P.n0 = n0;
  P.numLevels = numLevels;
  P.maxBox = maxBox;
  P.blockFactor = blockFactor;
  P.fillRatio = fillRatio;
  P.opType = opType;
  P.alpha = alpha;
  P.beta = beta;
  P.seed = seed;
  P.thresh = thresh;
  P.boxfile = args("boxfile", "");
  if (buildProblem(P) != 0) return 2;
  const int finest = P.finest, nlev = P.nlev;
  Vector<ProblemDomain>& domains = P.domains;
  Vector<Real>& dxs = P.dxs;
  Vector<DisjointBoxLayout>& grids = P.grids;
  if (argi("plansonly", 0)) {
    // Box layouts and copier plans only (no solve): <prefix>.plans, raw
    // little-endian int32, per level the exchange plan then (levels >= 1)
    // the coarsened-fine plan, each as a count followed by 14 ints per item
    // (from, to, fromRegion lo/hi, toRegion lo/hi).
    FILE* pf = std::fopen((out + ".plans").c_str(), "wb");
    auto put = [&](const Copier& c) {
      std::vector<int> v;
      for (CopyIterator it(c, CopyIterator::LOCAL); it.ok(); ++it) {
        const MotionItem& m = it();
        v.push_back(m.fromIndex.intCode());
        v.push_back(m.toIndex.intCode());
        for (const Box* b : {&m.fromRegion, &m.toRegion}) {
          for (int d = 0; d < 3; ++d) v.push_back(b->smallEnd(d));
          for (int d = 0; d < 3; ++d) v.push_back(b->bigEnd(d));
        }
      }
      int n = (int)(v.size() / 14);
      std::fwrite(&n, sizeof(int), 1, pf);
      std::fwrite(v.data(), sizeof(int), v.size(), pf);
    };
    for (int l = 0; l < nlev; ++l) {
      Copier ex;
      ex.exchangeDefine(grids[l], IntVect::Unit);
      ex.trimEdges(grids[l], IntVect::Unit);
      put(ex);
      if (l > 0) {
        DisjointBoxLayout cf;
        coarsen(cf, grids[l], 2);
        Copier c;
        c.define(cf, grids[l - 1], IntVect::Zero);
        put(c);
      }
    }
    std::fclose(pf);
    std::printf("oracle: plans of %d levels\n", nlev);
    return 0;
  }
  Vector<LDF*>& phi = P.phi;
  Vector<LDF*>& rhs = P.rhs;
  Vector<RefCountedPtr<LDF> >& aCoef = P.aCoef;
  Vector<RefCountedPtr<LevelData<FluxBox> > >& bCoef = P.bCoef;

  // Solver.
  Vector<DisjointBoxLayout> fgrids(nlev);
  for (int l = 0; l < nlev; ++l) fgrids[l] = grids[l];
  Vector<int> rr(nlev, 2);
  AMRLevelOpFactory<LDF>* factory = NULL;
  AMRPoissonOpFactory* pf = NULL;
  VCAMRPoissonOp2Factory* vf = NULL;
  if (opType == 0) {
    pf = new AMRPoissonOpFactory;
    pf->define(domains[0], fgrids, rr, dxs[0], &domainBC, alpha, beta);
    factory = pf;
  } else {
    vf = new VCAMRPoissonOp2Factory;
    vf->define(domains[0], fgrids, rr, dxs[0], &domainBC, alpha, aCoef, beta, bCoef);
    factory = vf;
  }
  AMRMultiGrid<LDF>* solver = new AMRMultiGrid<LDF>();
  BiCGStabSolver<LDF> bottomSolver;
  bottomSolver.m_verbosity = 0;
  solver->define(domains[0], *factory, &bottomSolver, nlev);
  solver->setSolverParameters(pre, post, bottom, 1, iterMax, eps, hang, 1e-30);
  solver->m_verbosity = argi("verbosity", 0);
  RefCountedPtr<AMRMultiGridInspector<LDF> > insp(new ResidualRecorder);
  ResidualRecorder* rec = static_cast<ResidualRecorder*>(&(*insp));

  double seconds = 0, tstart = 0, tend = 0;
  for (int rep = 0; rep < repeat; ++rep) {
    rec->norms.clear();
    rec->stamps.clear();
    if (rep == 0) solver->addInspector(insp);
    auto t0 = std::chrono::steady_clock::now();
    solver->solve(phi, rhs, finest, 0, true);
    auto t1 = std::chrono::steady_clock::now();
    tstart = std::chrono::duration<double>(t0.time_since_epoch()).count();
    tend = std::chrono::duration<double>(t1.time_since_epoch()).count();
    seconds += std::chrono::duration<double>(t1 - t0).count();
    // Per-repeat record for the CPU timing runs: total, set-up part and
    // per-iteration parts of this solve.
    std::vector<double> its;
    for (size_t i = 0; i < rec->stamps.size(); ++i)
      its.push_back((i + 1 < rec->stamps.size() ? rec->stamps[i + 1] : tend) - rec->stamps[i]);
    std::printf("repeat %d seconds %.9g setup %.9g iterations", rep, std::chrono::duration<double>(t1 - t0).count(),
                rec->stamps.empty() ? 0.0 : rec->stamps[0] - tstart);
    for (double t : its) std::printf(" %.9g", t);
    std::printf("\n");
    std::fflush(stdout);
  }
  int exitStatus = solver->m_exitStatus;
  double finalNorm = solver->computeAMRResidual(phi, rhs, finest, 0);
  rec->norms.push_back(finalNorm);

  // Exchange plans and coarsened-fine copy plans for the geometry checks.
  FILE* js = std::fopen((out + ".json").c_str(), "w");
  std::fprintf(js, "{\n\"n0\": %d, \"levels\": %d, \"maxbox\": %d, \"block\": %d, \"fill\": %.17g,\n", n0,
               nlev, maxBox, blockFactor, fillRatio);
  std::fprintf(js, "\"bc\": \"%s\",\n", faceBCString().c_str());
  std::fprintf(js, "\"op\": %d, \"alpha\": %.17g, \"beta\": %.17g, \"seed\": %llu, \"thresh\": %.17g,\n", opType,
               alpha, beta, seed, thresh);
  std::fprintf(js, "\"pre\": %d, \"post\": %d, \"bottom\": %d, \"iters\": %d, \"eps\": %.17g, \"hang\": %.17g,\n",
               pre, post, bottom, iterMax, eps, hang);
  std::fprintf(js, "\"exit_status\": %d, \"seconds_per_solve\": %.9g,\n", exitStatus, seconds / repeat);
  // Wall time of the last solve split into: start -> first iteration (set-up
  // and initial residual), each V-cycle iteration, and the tail.
  std::fprintf(js, "\"iteration_seconds\": [");
  for (size_t i = 0; i < rec->stamps.size(); ++i) {
    double t = (i + 1 < rec->stamps.size() ? rec->stamps[i + 1] : tend) - rec->stamps[i];
    std::fprintf(js, "%s%.9g", i ? "," : "", t);
  }
  std::fprintf(js, "],\n\"setup_seconds\": %.9g,\n", rec->stamps.empty() ? 0.0 : rec->stamps[0] - tstart);
  std::fprintf(js, "\"residual_history\": [");
  for (size_t i = 0; i < rec->norms.size(); ++i) std::fprintf(js, "%s%.17g", i ? "," : "", rec->norms[i]);
  std::fprintf(js, "],\n\"boxes\": [");
  for (int l = 0; l < nlev; ++l) {
    std::fprintf(js, "%s[", l ? "," : "");
    int ib = 0;
    for (LayoutIterator lit = grids[l].layoutIterator(); lit.ok(); ++lit, ++ib) {
      if (ib) std::fprintf(js, ",");
      writeBox(js, grids[l][lit]);
    }
    std::fprintf(js, "]");
  }
  std::fprintf(js, "],\n\"exchange_plans\": [");
  for (int l = 0; l < nlev; ++l) {
    Copier ex;
    ex.exchangeDefine(grids[l], IntVect::Unit);
    ex.trimEdges(grids[l], IntVect::Unit);
    std::fprintf(js, "%s", l ? "," : "");
    writeCopier(js, ex);
  }
  std::fprintf(js, "],\n\"coarsened_fine_plans\": [");
  for (int l = 1; l < nlev; ++l) {
    DisjointBoxLayout cf;
    coarsen(cf, grids[l], 2);
    Copier c;
    c.define(cf, grids[l - 1], IntVect::Zero);
    std::fprintf(js, "%s", l > 1 ? "," : "");
    writeCopier(js, c);
  }
  std::fprintf(js, "]\n}\n");
  std::fclose(js);

  if (dumpPhi) {
    FILE* bin = std::fopen((out + ".bin").c_str(), "wb");
    for (int l = 0; l < nlev; ++l) {
      for (LayoutIterator lit = grids[l].layoutIterator(); lit.ok(); ++lit) {
        DataIndex di(lit());
        writeFab(bin, (*rhs[l])[di], grids[l][lit]);
      }
      for (LayoutIterator lit = grids[l].layoutIterator(); lit.ok(); ++lit) {
        DataIndex di(lit());
        writeFab(bin, (*phi[l])[di], grids[l][lit]);
      }
      if (opType == 1) {
        for (LayoutIterator lit = grids[l].layoutIterator(); lit.ok(); ++lit) {
          DataIndex di(lit());
          writeFab(bin, (*aCoef[l])[di], grids[l][lit]);
        }
        for (int d = 0; d < 3; ++d)
          for (LayoutIterator lit = grids[l].layoutIterator(); lit.ok(); ++lit) {
            DataIndex di(lit());
            const FArrayBox& b = (*bCoef[l])[di][d];
            writeFab(bin, b, b.box());
          }
      }
    }
    std::fclose(bin);
  }

  for (int l = 0; l < nlev; ++l) {
    delete phi[l];
    delete rhs[l];
  }
  delete solver;
  delete factory;
  std::printf("oracle: levels=%d exit=%d iters=%zu r0=%.6e rfinal=%.6e seconds=%.4f\n", nlev, exitStatus,
              rec->norms.size() - 1, rec->norms.front(), rec->norms.back(), seconds / repeat);
  return 0;
}
