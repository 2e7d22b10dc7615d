// ORACLE — test infrastructure only.
//
// The drop-in check: a Chombo program solves the same seeded hierarchy twice
// through the same API, once with the reference's AMRMultiGrid over
// AMRPoissonOp / VCAMRPoissonOp2 on the CPU and once with
// cmg_chombo::GpuAMRMultiGrid over the GPU factories (include/cmg_chombo.H,
// libcmg.so), and prints one JSON line comparing the two: exit status,
// iteration count, residual histories and phi on every level.
//
// Usage: dropin key=value ...   (n0 levels maxbox block op alpha beta seed
// pre post bottom iters eps hang, as for cmg_oracle; bicgstab=1 mgiters
// mgsmooth imax eps for the BiCGStab over MultilevelLinearOp path; heat=1
// (backward Euler) or heat=2 (TGA) with dt steps for the heat solvers;
// fineinterp=1 (interpToFine) or 2 (pwcinterpToFine) for FineInterp)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

#include "AMRMultiGrid.H"
#include "AMRPoissonOp.H"
#include "AMRTGA.H"
#include "BackwardEuler.H"
#include "BiCGStabSolver.H"
#include "FineInterp.H"
#include "MultilevelLinearOp.H"
#include "VCAMRPoissonOp2.H"
#include "cmg_chombo.H"
#include "problem.H"

static std::map<std::string, std::string> g_args;
static double argd(const char* k, double d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? d : std::atof(it->second.c_str());
}

static double phiDeviation(const OracleProblem& P, const Vector<LDF*>& phiGpu) {
  double maxRel = 0;
  for (int l = 0; l < P.nlev; ++l) {
    double scale = 0, diff = 0;
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) {
      const Box& b = P.grids[l][dit()];
      for (BoxIterator bit(b); bit.ok(); ++bit) {
        scale = std::max(scale, std::fabs((*P.phi[l])[dit](bit(), 0)));
        diff = std::max(diff, std::fabs((*P.phi[l])[dit](bit(), 0) - (*phiGpu[l])[dit](bit(), 0)));
      }
    }
    maxRel = std::max(maxRel, scale > 0 ? diff / scale : diff);
  }
  return maxRel;
}

// The variable-coefficient example's solve path (VCPoissonSolve.cpp:146-183):
// the reference's BiCGStabSolver over MultilevelLinearOp on the CPU, then the
// same calls on cmg_chombo::GpuMultilevelLinearOp + GpuMultilevelBiCGStabSolver.
static int bicgstabCheck(OracleProblem& P, Vector<LDF*>& phiGpu, Vector<int>& rr) {
  const int nlev = P.nlev;
  const int mgIters = (int)argd("mgiters", 2), mgSmooth = (int)argd("mgsmooth", 4), imax = (int)argd("imax", 100);
  const Real eps = argd("eps", 1e-9);
  Vector<RealVect> dxv(nlev);
  for (int l = 0; l < nlev; ++l) dxv[l] = RealVect::Unit * P.dxs[l];
  RefCountedPtr<AMRLevelOpFactory<LDF> > factory;
  if (P.opType == 0) {
    AMRPoissonOpFactory* f = new AMRPoissonOpFactory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.beta);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  }
  for (int l = 0; l < nlev; ++l)
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) {
      (*P.phi[l])[dit()].setVal(0.0);
      (*phiGpu[l])[dit()].setVal(0.0);
    }
  MultilevelLinearOp<FArrayBox> mlOp;
  mlOp.m_num_mg_iterations = mgIters;
  mlOp.m_num_mg_smooth = mgSmooth;
  mlOp.define(P.grids, rr, P.domains, dxv, factory, 0);
  BiCGStabSolver<Vector<LDF*> > cpu;
  cpu.define(&mlOp, false);
  cpu.m_verbosity = 0;
  cpu.m_normType = 0;
  cpu.m_eps = eps;
  cpu.m_imax = imax;
  cpu.solve(P.phi, P.rhs);

  cmg_chombo::GpuMultilevelLinearOp gop;
  gop.m_num_mg_iterations = mgIters;
  gop.m_num_mg_smooth = mgSmooth;
  if (P.opType == 0) {
    cmg_chombo::GpuAMRPoissonOpFactory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.beta);
    gop.define(P.grids, rr, P.domains, dxv, f, 0);
  } else {
    cmg_chombo::GpuVCAMRPoissonOp2Factory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    gop.define(P.grids, rr, P.domains, dxv, f, 0);
  }
  cmg_chombo::GpuMultilevelBiCGStabSolver gpu;
  gpu.define(&gop, false);
  gpu.m_verbosity = 0;
  gpu.m_normType = 0;
  gpu.m_eps = eps;
  gpu.m_imax = imax;
  gpu.solve(phiGpu, P.rhs);
  std::printf("{\"levels\": %d, \"cpu_exit\": %d, \"gpu_exit\": %d, \"cpu_iters\": %d, \"gpu_iters\": %d, "
              "\"cpu_r0\": %.17g, \"gpu_r0\": %.17g, \"cpu_rfinal\": %.17g, \"gpu_rfinal\": %.17g, "
              "\"phi_rel_dev\": %.3e}\n",
              nlev, cpu.m_exitStatus, gpu.m_exitStatus, cpu.m_iter, gpu.m_iter, cpu.m_initial_residual,
              gpu.m_initial_residual, cpu.m_residual, gpu.m_residual, phiDeviation(P, phiGpu));
  for (int l = 0; l < nlev; ++l) {
    delete phiGpu[l];
    delete P.phi[l];
    delete P.rhs[l];
  }
  return 0;
}

// The heat solvers (BackwardEuler, AMRTGA) on the CPU and through
// cmg_chombo::GpuBackwardEuler / GpuAMRTGA with the same calls: the initial
// state and the source are the seeded right-hand side (with one ghost layer).
static int heatCheck(OracleProblem& P, Vector<LDF*>& phiGpu, Vector<int>& rr, bool tga) {
  const int nlev = P.nlev, lmax = P.finest;
  const int steps = (int)argd("steps", 2);
  const Real dt = argd("dt", 1e-3);
  const int pre = (int)argd("pre", 4), post = (int)argd("post", 4), bottom = (int)argd("bottom", 4);
  const Real eps = argd("eps", 1e-10), hang = argd("hang", 1e-10);
  Vector<LDF*> phiOld(nlev), phiNew(nlev), src(nlev), gOld(nlev);
  for (int l = 0; l < nlev; ++l) {
    phiOld[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    phiNew[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    src[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    gOld[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) {
      for (LDF* f : {phiOld[l], phiNew[l], src[l], gOld[l], phiGpu[l]}) (*f)[dit()].setVal(0.0);
      (*phiOld[l])[dit()].copy((*P.rhs[l])[dit()], P.grids[l][dit()]);
      (*gOld[l])[dit()].copy((*P.rhs[l])[dit()], P.grids[l][dit()]);
      (*src[l])[dit()].copy((*P.rhs[l])[dit()], P.grids[l][dit()]);
    }
  }
  RefCountedPtr<AMRLevelOpFactory<LDF> > factory;
  if (P.opType == 0) {
    AMRPoissonOpFactory* f = new AMRPoissonOpFactory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.beta);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  }
  BiCGStabSolver<LDF> bottomSolver;
  bottomSolver.m_verbosity = 0;
  RefCountedPtr<AMRMultiGrid<LDF> > cpu(new AMRMultiGrid<LDF>());
  cpu->define(P.domains[0], *factory, &bottomSolver, nlev);
  cpu->setSolverParameters(pre, post, bottom, 1, 100, eps, hang, 1e-30);
  cpu->m_verbosity = 0;
  if (tga) {
    cpu->init(phiNew, src, lmax, 0);
    cpu->setBottomSolver(lmax, 0);
    AMRTGA<LDF> t(cpu, *factory, P.domains[0], rr, nlev, 0);
    for (int n = 0; n < steps; ++n) {
      t.oneStep(phiNew, phiOld, src, dt, 0, lmax, 0.0);
      std::swap(phiNew, phiOld);
    }
  } else {
    BackwardEuler be(cpu, *factory, P.domains[0], rr, nlev, 0);
    for (int n = 0; n < steps; ++n) {
      be.oneStep(phiNew, phiOld, src, dt, 0, lmax, false);
      std::swap(phiNew, phiOld);
    }
  }

  RefCountedPtr<cmg_chombo::GpuAMRMultiGrid> gpu(new cmg_chombo::GpuAMRMultiGrid());
  BiCGStabSolver<LDF> gpuBottom;
  cmg_chombo::GpuAMRPoissonOpFactory pf;
  cmg_chombo::GpuVCAMRPoissonOp2Factory vf;
  if (P.opType == 0) {
    pf.define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.beta);
    gpu->define(P.domains[0], pf, &gpuBottom, nlev);
  } else {
    vf.define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    gpu->define(P.domains[0], vf, &gpuBottom, nlev);
  }
  gpu->setSolverParameters(pre, post, bottom, 1, 100, eps, hang, 1e-30);
  if (tga) {
    cmg_chombo::GpuAMRTGA t(gpu, pf, P.domains[0], rr, nlev, 0);
    for (int n = 0; n < steps; ++n) {
      t.oneStep(phiGpu, gOld, src, dt, 0, lmax, 0.0);
      std::swap(phiGpu, gOld);
    }
  } else {
    cmg_chombo::GpuBackwardEuler be(gpu, pf, P.domains[0], rr, nlev, 0);
    for (int n = 0; n < steps; ++n) {
      be.oneStep(phiGpu, gOld, src, dt, 0, lmax, false);
      std::swap(phiGpu, gOld);
    }
  }
  // the latest states are in phiOld (CPU) and gOld (GPU)
  for (int l = 0; l < nlev; ++l) delete P.phi[l];
  for (int l = 0; l < nlev; ++l) P.phi[l] = phiOld[l];
  std::printf("{\"levels\": %d, \"scheme\": \"%s\", \"cpu_exit\": %d, \"gpu_exit\": %d, "
              "\"phi_rel_dev\": %.3e}\n",
              nlev, tga ? "tga" : "euler", cpu->m_exitStatus, gpu->m_exitStatus, phiDeviation(P, gOld));
  return 0;
}

// FineInterp on the CPU and cmg_chombo::GpuFineInterp with the same calls:
// every level above 0 is filled from the level below (interpToFine, or
// pwcinterpToFine with fineinterp=2), the coarse data being the seeded
// right-hand side; the fine data must agree bit for bit.
static int fineInterpCheck(OracleProblem& P, bool pwc) {
  double maxDiff = 0.0;
  long cells = 0;
  for (int l = 1; l < P.nlev; ++l) {
    LDF cpuFine(P.grids[l], 1, IntVect::Unit), gpuFine(P.grids[l], 1, IntVect::Unit);
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) {
      cpuFine[dit()].setVal(0.0);
      gpuFine[dit()].setVal(0.0);
    }
    FineInterp cpu(P.grids[l], 1, 2, P.domains[l]);
    cmg_chombo::GpuFineInterp gpu(P.grids[l], 1, 2, P.domains[l]);
    if (pwc) {
      cpu.pwcinterpToFine(cpuFine, *P.rhs[l - 1]);
      gpu.pwcinterpToFine(gpuFine, *P.rhs[l - 1]);
    } else {
      cpu.interpToFine(cpuFine, *P.rhs[l - 1]);
      gpu.interpToFine(gpuFine, *P.rhs[l - 1]);
      gpu.interpToFine(gpuFine, *P.rhs[l - 1]);  // the kept device plan
    }
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) {
      const Box& b = P.grids[l][dit()];
      for (BoxIterator bit(b); bit.ok(); ++bit) {
        maxDiff = std::max(maxDiff, std::fabs(cpuFine[dit()](bit(), 0) - gpuFine[dit()](bit(), 0)));
        ++cells;
      }
    }
  }
  std::printf("{\"fineinterp\": %d, \"levels\": %d, \"cells\": %ld, \"max_abs_diff\": %.17g}\n", pwc ? 2 : 1,
              P.nlev, cells, maxDiff);
  return 0;
}

int main(int argc, char** argv) {
  for (int a = 1; a < argc; ++a) {
    const char* eq = std::strchr(argv[a], '=');
    if (eq) g_args[std::string(argv[a], eq - argv[a])] = std::string(eq + 1);
  }
  OracleProblem P;
  P.n0 = (int)argd("n0", 16);
  P.numLevels = (int)argd("levels", 3);
  P.maxBox = (int)argd("maxbox", 8);
  P.blockFactor = (int)argd("block", 4);
  P.opType = (int)argd("op", 1);
  P.alpha = argd("alpha", 1.0);
  P.beta = argd("beta", -1.0);
  P.seed = (unsigned long long)argd("seed", 20261203.0);
  if (buildProblem(P) != 0) return 2;
  const int pre = (int)argd("pre", 4), post = (int)argd("post", 4), bottom = (int)argd("bottom", 4);
  const int iters = (int)argd("iters", 100);
  const Real eps = argd("eps", 1e-10), hang = argd("hang", 1e-10);
  const int nlev = P.nlev, lmax = P.finest;

  Vector<LDF*> phiGpu(nlev);
  for (int l = 0; l < nlev; ++l) phiGpu[l] = new LDF(P.grids[l], 1, IntVect::Unit);
  Vector<int> rr(nlev, 2);
  if (argd("bicgstab", 0) != 0) return bicgstabCheck(P, phiGpu, rr);
  if (argd("heat", 0) != 0) return heatCheck(P, phiGpu, rr, argd("heat", 0) == 2);
  if (argd("fineinterp", 0) != 0) return fineInterpCheck(P, argd("fineinterp", 0) == 2);

  // Reference: CPU AMRMultiGrid.
  RefCountedPtr<AMRLevelOpFactory<LDF> > factory;
  if (P.opType == 0) {
    AMRPoissonOpFactory* f = new AMRPoissonOpFactory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.beta);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  }
  BiCGStabSolver<LDF> bottomSolver;
  bottomSolver.m_verbosity = 0;
  AMRMultiGrid<LDF> cpu;
  cpu.define(P.domains[0], *factory, &bottomSolver, nlev);
  cpu.setSolverParameters(pre, post, bottom, 1, iters, eps, hang, 1e-30);
  cpu.m_verbosity = 0;
  RefCountedPtr<AMRMultiGridInspector<LDF> > insp(new ResidualRecorder);
  cpu.addInspector(insp);
  cpu.solve(P.phi, P.rhs, lmax, 0, true);
  ResidualRecorder* rec = static_cast<ResidualRecorder*>(&(*insp));
  rec->norms.push_back(cpu.computeAMRResidual(P.phi, P.rhs, lmax, 0));

  // The same calls on the GPU drop-in.
  cmg_chombo::GpuAMRMultiGrid gpu;
  BiCGStabSolver<LDF> gpuBottom;
  if (P.opType == 0) {
    cmg_chombo::GpuAMRPoissonOpFactory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.beta);
    gpu.define(P.domains[0], f, &gpuBottom, nlev);
  } else {
    cmg_chombo::GpuVCAMRPoissonOp2Factory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &dirichletBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    gpu.define(P.domains[0], f, &gpuBottom, nlev);
  }
  gpu.setSolverParameters(pre, post, bottom, 1, iters, eps, hang, 1e-30);
  gpu.solve(phiGpu, P.rhs, lmax, 0, true);
  const Real gpuFinal = gpu.computeAMRResidual(phiGpu, P.rhs, lmax, 0);

  double maxRel = 0, maxHist = 0;
  for (int l = 0; l < nlev; ++l) {
    double scale = 0, diff = 0;
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) {
      const Box& b = P.grids[l][dit()];
      for (BoxIterator bit(b); bit.ok(); ++bit) {
        scale = std::max(scale, std::fabs((*P.phi[l])[dit](bit(), 0)));
        diff = std::max(diff, std::fabs((*P.phi[l])[dit](bit(), 0) - (*phiGpu[l])[dit](bit(), 0)));
      }
    }
    maxRel = std::max(maxRel, scale > 0 ? diff / scale : diff);
  }
  const std::vector<double>& gh = gpu.residualHistory();
  const bool sameLen = gh.size() == rec->norms.size();
  if (sameLen)
    for (size_t i = 0; i < gh.size(); ++i) maxHist = std::max(maxHist, std::fabs(gh[i] - rec->norms[i]) / rec->norms[0]);
  std::printf("{\"levels\": %d, \"cpu_exit\": %d, \"gpu_exit\": %d, \"cpu_iters\": %d, \"gpu_iters\": %d, "
              "\"same_history_length\": %s, \"history_dev\": %.3e, \"phi_rel_dev\": %.3e, "
              "\"gpu_final_residual\": %.17g, \"gpu_history_last\": %.17g}\n",
              nlev, cpu.m_exitStatus, gpu.m_exitStatus, (int)rec->norms.size() - 1, gpu.iterations(),
              sameLen ? "true" : "false", maxHist, maxRel, gpuFinal, gh.empty() ? -1.0 : gh.back());
  for (int l = 0; l < nlev; ++l) {
    delete phiGpu[l];
    delete P.phi[l];
    delete P.rhs[l];
  }
  return 0;
}
