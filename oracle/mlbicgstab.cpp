// ORACLE — test infrastructure only.  Never linked into the product.
//
// Runs the reference's BiCGStabSolver<Vector<LevelData<FArrayBox>*>>
// (lib/src/AMRElliptic/BiCGStabSolver.H:199-515) over its
// MultilevelLinearOp<FArrayBox> (MultilevelLinearOp.H, MultilevelLinearOpI.H)
// preconditioned by AMR multigrid V-cycles, set up as the variable-coefficient
// example does (releasedExamples/AMRPoisson/execVariableCoefficient/
// VCPoissonSolve.cpp:146-183: lBase 0, m_num_mg_iterations, m_num_mg_smooth,
// normType 0, m_eps, m_imax), on the seeded synthetic hierarchies of the
// benchmark workloads (problem.H), and dumps what the GPU path is checked
// against: exit status, iteration count, initial and final residual norms,
// and phi on every level.
//
// Usage: cmg_oracle_mlbicgstab key=value ... out=<prefix>
//   n0 levels maxbox block fill op alpha beta seed thresh (as cmg_oracle)
//   mgiters=1 mgsmooth=4 eps=1e-9 imax=100 [boxfile=<file> as cmg_oracle]
// Writes <prefix>.json and <prefix>.bin (per level, per box in layout order,
// valid cells x-fastest: phi).

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "AMRPoissonOp.H"
#include "BCFunc.H"
#include "BiCGStabSolver.H"
#include "MultilevelLinearOp.H"
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
  P.alpha = argd("alpha", 0.0);
  P.beta = argd("beta", 1.0);
  P.seed = (unsigned long long)argd("seed", 20261203.0);
  P.thresh = argd("thresh", 0.1);
  if (g_args.count("boxfile")) P.boxfile = g_args["boxfile"];
  const int mgIters = argi("mgiters", 1), mgSmooth = argi("mgsmooth", 4), imax = argi("imax", 100);
  const Real eps = argd("eps", 1e-9);
  const std::string out = g_args.count("out") ? g_args["out"] : std::string("mlbicgstab_out");
  if (buildProblem(P) != 0) return 2;
  const int nlev = P.nlev;

  Vector<DisjointBoxLayout> grids(nlev);
  Vector<ProblemDomain> domains(nlev);
  Vector<RealVect> dxv(nlev);
  for (int l = 0; l < nlev; ++l) {
    grids[l] = P.grids[l];
    domains[l] = P.domains[l];
    dxv[l] = RealVect::Unit * P.dxs[l];
  }
  Vector<int> rr(nlev, 2);
  RefCountedPtr<AMRLevelOpFactory<LDF> > factory;
  if (P.opType == 0) {
    AMRPoissonOpFactory* pf = new AMRPoissonOpFactory;
    pf->define(domains[0], grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(pf);
  } else {
    VCAMRPoissonOp2Factory* vf = new VCAMRPoissonOp2Factory;
    vf->define(domains[0], grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(vf);
  }
  // Zero initial guess, ghost cells included (VCPoissonSolve.cpp:131-134).
  for (int l = 0; l < nlev; ++l)
    for (DataIterator dit = grids[l].dataIterator(); dit.ok(); ++dit) (*P.phi[l])[dit()].setVal(0.0);
  MultilevelLinearOp<FArrayBox> mlOp;
  mlOp.m_num_mg_iterations = mgIters;
  mlOp.m_num_mg_smooth = mgSmooth;
  mlOp.m_preCondSolverDepth = -1;
  mlOp.define(grids, rr, domains, dxv, factory, 0);

  BiCGStabSolver<Vector<LDF*> > solver;
  solver.define(&mlOp, false);
  solver.m_verbosity = 0;
  solver.m_normType = 0;
  solver.m_eps = eps;
  solver.m_imax = imax;
  const auto t0 = std::chrono::steady_clock::now();
  solver.solve(P.phi, P.rhs);
  const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  FILE* js = std::fopen((out + ".json").c_str(), "w");
  std::fprintf(js, "{\"exit_status\": %d, \"iterations\": %d, \"initial_residual\": %.17g, \"final_residual\": %.17g,"
                   " \"seconds\": %.9g, \"mgiters\": %d, \"mgsmooth\": %d, \"eps\": %.17g, \"imax\": %d, \"boxes\": [",
               solver.m_exitStatus, solver.m_iter, solver.m_initial_residual, solver.m_residual, seconds, mgIters,
               mgSmooth, eps, imax);
  for (int l = 0; l < nlev; ++l) {
    std::fprintf(js, "%s[", l ? "," : "");
    int ib = 0;
    for (LayoutIterator lit = grids[l].layoutIterator(); lit.ok(); ++lit, ++ib) {
      const Box& b = grids[l][lit];
      std::fprintf(js, "%s[%d,%d,%d,%d,%d,%d]", ib ? "," : "", b.smallEnd(0), b.smallEnd(1), b.smallEnd(2),
                   b.bigEnd(0), b.bigEnd(1), b.bigEnd(2));
    }
    std::fprintf(js, "]");
  }
  std::fprintf(js, "]}\n");
  std::fclose(js);
  FILE* bin = std::fopen((out + ".bin").c_str(), "wb");
  for (int l = 0; l < nlev; ++l)
    for (LayoutIterator lit = grids[l].layoutIterator(); lit.ok(); ++lit) {
      const Box& b = grids[l][lit];
      const FArrayBox& fab = (*P.phi[l])[DataIndex(lit())];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
          for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) {
            double v = fab(IntVect(i, j, k), 0);
            std::fwrite(&v, sizeof(double), 1, bin);
          }
    }
  std::fclose(bin);
  std::printf("mlbicgstab: levels=%d exit=%d iters=%d r0=%.6e rfinal=%.6e seconds=%.3f\n", nlev, solver.m_exitStatus,
              solver.m_iter, solver.m_initial_residual, solver.m_residual, seconds);
  return 0;
}
