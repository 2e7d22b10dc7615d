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
// fineinterp=1 (interpToFine) or 2 (pwcinterpToFine) for FineInterp; ops=1
// for the operator-by-operator comparison of the reference's operators with
// the GPU AMRLevelOps; amrmg=1 for the reference's AMRMultiGrid over the
// reference factory and over the GPU factory, amrmg=1 fas=1 for its
// AMRFASMultiGrid the same way; bc=<six letters D/N> sets the homogeneous
// Dirichlet / Neumann type of each domain face; bcprobe=1 prints the face
// types the GPU factory reads off that BC function; badbc=1 hands an
// inhomogeneous Dirichlet BC to the GPU factory, which must refuse it)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

#include "AMRFASMultiGrid.H"
#include "AMRMultiGrid.H"
#include "AMRPoissonOp.H"
#include "AMRTGA.H"
#include "BackwardEuler.H"
#include "BiCGStabSolver.H"
#include "FineInterp.H"
#include "MultilevelLinearOp.H"
#include "QuadCFInterp.H"
#include "RelaxSolver.H"
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
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
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
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    gop.define(P.grids, rr, P.domains, dxv, f, 0);
  } else {
    cmg_chombo::GpuVCAMRPoissonOp2Factory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
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
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
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
    pf.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    gpu->define(P.domains[0], pf, &gpuBottom, nlev);
  } else {
    vf.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
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

// A seeded field over every FAB cell of a level (ghost cells included), so
// that the operators read the same inputs wherever they look.
static void seededField(LDF& f, Real dx, const cmg_synth::Bumps& bumps, unsigned salt) {
  for (DataIterator dit = f.dataIterator(); dit.ok(); ++dit) {
    FArrayBox& fab = f[dit()];
    for (BoxIterator bit(fab.box()); bit.ok(); ++bit) {
      const IntVect iv = bit();
      unsigned h = (unsigned)(iv[0] * 73856093) ^ (unsigned)(iv[1] * 19349663) ^ (unsigned)(iv[2] * 83492791) ^ salt;
      h = h * 2654435761u;
      fab(iv, 0) = bumps.eval((iv[0] + 0.5) * dx, (iv[1] + 0.5) * dx, (iv[2] + 0.5) * dx) + 1e-3 * (double)(h % 1000) / 1000.0;
    }
  }
}

static void copyAll(LDF& dst, const LDF& src) {
  for (DataIterator dit = src.dataIterator(); dit.ok(); ++dit) dst[dit()].copy(src[dit()]);
}

struct OpDiff {
  double maxAbs = 0;
  long ndiff = 0, cells = 0;
};

// Cells of the next finer level's coarsened boxes (covered cells): skipped
// by validDiff when g_skipCovered is set.
static const DisjointBoxLayout* g_covered = nullptr;
static bool g_skipCovered = false;
static int g_detail = 0;

static OpDiff validDiff(const LDF& a, const LDF& b) {
  OpDiff d;
  int shown = 0;
  for (DataIterator dit = a.dataIterator(); dit.ok(); ++dit) {
    const Box& bx = a.disjointBoxLayout()[dit()];
    for (BoxIterator bit(bx); bit.ok(); ++bit) {
      if (g_skipCovered && g_covered) {
        bool cov = false;
        for (LayoutIterator lit = g_covered->layoutIterator(); lit.ok() && !cov; ++lit)
          cov = (*g_covered)[lit()].contains(bit());
        if (cov) continue;
      }
      const double x = a[dit()](bit(), 0), y = b[dit()](bit(), 0);
      ++d.cells;
      if (x != y && !(x != x && y != y)) {
        ++d.ndiff;
        d.maxAbs = std::max(d.maxAbs, std::fabs(x - y));
        if (g_detail && shown < g_detail) {
          bool cov = false;
          if (g_covered)
            for (LayoutIterator lit = g_covered->layoutIterator(); lit.ok(); ++lit)
              cov = cov || (*g_covered)[lit()].contains(bit());
          std::fprintf(stderr, "  cell (%d,%d,%d) covered=%d ref=%.17g gpu=%.17g\n", bit()[0], bit()[1], bit()[2],
                       (int)cov, x, y);
          ++shown;
        }
      }
    }
  }
  return d;
}

// Operator-by-operator parity: the reference's AMRPoissonOp / VCAMRPoissonOp2
// and the GPU AMRLevelOps (cmg_chombo::GpuAMRPoissonOp) built by their
// factories from the same grids and coefficients get identical LevelData
// inputs, one method at a time, and every valid cell of every output is
// compared bit for bit.  One JSON line: per (level, method) the count of
// differing cells and the largest difference.
static int opsCheck(OracleProblem& P, Vector<int>& rr) {
  const int nlev = P.nlev;
  RefCountedPtr<AMRLevelOpFactory<LDF> > refFactory;
  if (P.opType == 0) {
    AMRPoissonOpFactory* f = new AMRPoissonOpFactory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    refFactory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    refFactory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  }
  cmg_chombo::GpuAMRPoissonOpFactory gpf;
  cmg_chombo::GpuVCAMRPoissonOp2Factory gvf;
  cmg_chombo::GpuOpFactoryBase* gpuFactory = &gpf;
  if (P.opType == 0)
    gpf.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
  else {
    gvf.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    gpuFactory = &gvf;
  }
  std::vector<AMRLevelOp<LDF>*> ro(nlev), go(nlev);
  for (int l = 0; l < nlev; ++l) {
    ro[l] = refFactory->AMRnewOp(P.domains[l]);
    go[l] = gpuFactory->AMRnewOp(P.domains[l]);
  }
  cmg_synth::Problem prob(P.seed);
  std::vector<LDF*> phi(nlev), rhs(nlev);
  for (int l = 0; l < nlev; ++l) {
    phi[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    rhs[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    seededField(*phi[l], P.dxs[l], prob.bumps, 17u);
    seededField(*rhs[l], P.dxs[l], prob.bumps, 91u);
  }
  std::string json = "{\"ops\": [";
  bool first = true;
  auto report = [&](int lev, const char* name, const OpDiff& d) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s{\"level\": %d, \"op\": \"%s\", \"cells\": %ld, \"ndiff\": %ld, \"max_abs\": %.3e}",
                  first ? "" : ", ", lev, name, d.cells, d.ndiff, d.maxAbs);
    json += buf;
    first = false;
  };
  auto scalar = [&](int lev, const char* name, double a, double b) {
    OpDiff d;
    d.cells = 1;
    if (a != b) {
      d.ndiff = 1;
      d.maxAbs = std::fabs(a - b);
    }
    report(lev, name, d);
  };
  // out_ref / out_gpu start as the same copy; each side runs fn on its op
  // with its own copies of the inputs.
  struct Pair {
    LDF r, g;
  };
  auto mk = [&](const DisjointBoxLayout& dbl, const LDF* init) {
    Pair* p = new Pair;
    p->r.define(dbl, 1, IntVect::Unit);
    p->g.define(dbl, 1, IntVect::Unit);
    for (DataIterator dit = dbl.dataIterator(); dit.ok(); ++dit) {
      if (init) {
        p->r[dit()].copy((*init)[dit()]);
        p->g[dit()].copy((*init)[dit()]);
      } else {
        p->r[dit()].setVal(0.0);
        p->g[dit()].setVal(0.0);
      }
    }
    return p;
  };
  for (int l = 0; l < nlev; ++l) {
    const DisjointBoxLayout& g = P.grids[l];
    {  // LinearOp::residual, homogeneous and not
      for (int homog = 0; homog <= 1; ++homog) {
        Pair *ph = mk(g, phi[l]), *out = mk(g, nullptr);
        ro[l]->residual(out->r, ph->r, *rhs[l], homog);
        go[l]->residual(out->g, ph->g, *rhs[l], homog);
        report(l, homog ? "residual_homog" : "residual", validDiff(out->r, out->g));
        delete ph;
        delete out;
      }
    }
    {
      Pair *ph = mk(g, phi[l]), *out = mk(g, nullptr);
      ro[l]->applyOp(out->r, ph->r, true);
      go[l]->applyOp(out->g, ph->g, true);
      report(l, "applyOp", validDiff(out->r, out->g));
      delete ph;
      delete out;
    }
    {
      Pair* ph = mk(g, phi[l]);
      ro[l]->relax(ph->r, *rhs[l], 2);
      go[l]->relax(ph->g, *rhs[l], 2);
      report(l, "relax2", validDiff(ph->r, ph->g));
      delete ph;
    }
    {
      Pair* ph = mk(g, phi[l]);
      ro[l]->preCond(ph->r, *rhs[l]);
      go[l]->preCond(ph->g, *rhs[l]);
      report(l, "preCond", validDiff(ph->r, ph->g));
      delete ph;
    }
    {
      const bool hasC = l > 0, hasF = l + 1 < nlev;
      LDF empty;
      const LDF& pc = hasC ? *phi[l - 1] : empty;
      const LDF& pf = hasF ? *phi[l + 1] : empty;
      AMRLevelOp<LDF>* rf = hasF ? ro[l + 1] : nullptr;
      AMRLevelOp<LDF>* gf = hasF ? go[l + 1] : nullptr;
      // the operators write ghost cells of the finer and coarser phi: each
      // side gets its own copies
      Pair *pfc = hasF ? mk(P.grids[l + 1], phi[l + 1]) : nullptr, *pcc = hasC ? mk(P.grids[l - 1], phi[l - 1]) : nullptr;
      (void)pf;
      (void)pc;
      for (int form = 0; form < 2; ++form) {
        Pair *ph = mk(g, phi[l]), *out = mk(g, nullptr);
        if (hasC && hasF) {
          if (form == 0) {
            ro[l]->AMROperator(out->r, pfc->r, ph->r, pcc->r, true, rf);
            go[l]->AMROperator(out->g, pfc->g, ph->g, pcc->g, true, gf);
          } else {
            ro[l]->AMRResidual(out->r, pfc->r, ph->r, pcc->r, *rhs[l], true, rf);
            go[l]->AMRResidual(out->g, pfc->g, ph->g, pcc->g, *rhs[l], true, gf);
          }
        } else if (hasF) {
          if (form == 0) {
            ro[l]->AMROperatorNC(out->r, pfc->r, ph->r, true, rf);
            go[l]->AMROperatorNC(out->g, pfc->g, ph->g, true, gf);
          } else {
            ro[l]->AMRResidualNC(out->r, pfc->r, ph->r, *rhs[l], true, rf);
            go[l]->AMRResidualNC(out->g, pfc->g, ph->g, *rhs[l], true, gf);
          }
        } else if (hasC) {
          if (form == 0) {
            ro[l]->AMROperatorNF(out->r, ph->r, pcc->r, true);
            go[l]->AMROperatorNF(out->g, ph->g, pcc->g, true);
          } else {
            ro[l]->AMRResidualNF(out->r, ph->r, pcc->r, *rhs[l], true);
            go[l]->AMRResidualNF(out->g, ph->g, pcc->g, *rhs[l], true);
          }
        } else {
          delete ph;
          delete out;
          continue;
        }
        // The reference's flux register also adds into covered cells next to
        // the fine boundary (LevelFluxRegister::reflux adds the whole register
        // FABs); every caller discards those values (zeroCovered, or the
        // restricted fine residual written over them), so the operator is
        // compared on the valid cells not under the finer level.
        DisjointBoxLayout cov;
        if (hasF) coarsen(cov, P.grids[l + 1], 2);
        g_covered = hasF ? &cov : nullptr;
        g_skipCovered = true;
        g_detail = (int)argd("detail", 0);
        if (g_detail) std::fprintf(stderr, "level %d %s\n", l, form == 0 ? "AMROperator" : "AMRResidual");
        report(l, form == 0 ? "AMROperator" : "AMRResidual", validDiff(out->r, out->g));
        g_detail = 0;
        g_skipCovered = false;
        g_covered = nullptr;
        delete ph;
        delete out;
      }
      if (hasC) {
        // AMRRestrictS onto the coarsened-fine layout, then assignCopier onto
        // the coarse level (as AMRVCycle does).
        Pair *e = mk(g, phi[l]), *ec = mk(P.grids[l - 1], phi[l - 1]);
        LDF rr_, rg;
        ro[l]->createCoarsened(rr_, *rhs[l], 2);
        go[l]->createCoarsened(rg, *rhs[l], 2);
        LDF sr, sg;
        ro[l]->create(sr, *rhs[l]);
        go[l]->create(sg, *rhs[l]);
        ro[l]->AMRRestrictS(rr_, *rhs[l], e->r, ec->r, sr);
        go[l]->AMRRestrictS(rg, *rhs[l], e->g, ec->g, sg);
        report(l, "AMRRestrictS", validDiff(rr_, rg));
        Copier cr, cg;
        ro[l - 1]->buildCopier(cr, *rhs[l - 1], rr_);
        go[l - 1]->buildCopier(cg, *rhs[l - 1], rg);
        Pair* res = mk(P.grids[l - 1], rhs[l - 1]);
        ro[l - 1]->assignCopier(res->r, rr_, cr);
        go[l - 1]->assignCopier(res->g, rg, cg);
        report(l - 1, "assignCopier", validDiff(res->r, res->g));
        // zeroCovered of the coarse level under this one
        Pair* z = mk(P.grids[l - 1], rhs[l - 1]);
        ro[l - 1]->zeroCovered(z->r, rr_, cr);
        go[l - 1]->zeroCovered(z->g, rg, cg);
        report(l - 1, "zeroCovered", validDiff(z->r, z->g));
        delete res;
        delete z;
        // AMRProlongS and AMRUpdateResidual
        Pair* corr = mk(g, phi[l]);
        Copier rev = cr;
        rev.reverse();
        ro[l]->AMRProlongS(corr->r, ec->r, rr_, rev);
        go[l]->AMRProlongS(corr->g, ec->g, rg, rev);
        report(l, "AMRProlongS", validDiff(corr->r, corr->g));
        Pair* res2 = mk(g, rhs[l]);
        ro[l]->AMRUpdateResidual(res2->r, e->r, ec->r);
        go[l]->AMRUpdateResidual(res2->g, e->g, ec->g);
        report(l, "AMRUpdateResidual", validDiff(res2->r, res2->g));
        delete corr;
        delete res2;
        delete e;
        delete ec;
      }
      delete pfc;
      delete pcc;
    }
    if (l > 0) {  // QuadCFInterp::coarseFineInterp: every ghost cell of every FAB
      Pair* ph = mk(g, phi[l]);
      QuadCFInterp qcfi(g, &P.grids[l - 1], P.dxs[l], 2, 1, P.domains[l]);
      qcfi.coarseFineInterp(ph->r, *phi[l - 1]);
      static_cast<cmg_chombo::GpuAMRPoissonOp*>(go[l])->coarseFineInterp(ph->g, *phi[l - 1]);
      OpDiff d;
      int shown = 0;
      for (DataIterator dit = g.dataIterator(); dit.ok(); ++dit) {
        const Box& vb = g[dit()];
        for (BoxIterator bit(grow(vb, 1)); bit.ok(); ++bit) {
          if (vb.contains(bit())) continue;
          const double x = ph->r[dit()](bit(), 0), y = ph->g[dit()](bit(), 0);
          ++d.cells;
          if (x != y) {
            ++d.ndiff;
            d.maxAbs = std::max(d.maxAbs, std::fabs(x - y));
            if (shown++ < (int)argd("detail", 0))
              std::fprintf(stderr, "  cf ghost box %d (%d,%d,%d) ref=%.17g gpu=%.17g\n", (int)dit().intCode(), bit()[0],
                           bit()[1], bit()[2], x, y);
          }
        }
      }
      report(l, "coarseFineInterp", d);
      delete ph;
    }
    // LevelDataOps
    scalar(l, "norm0", ro[l]->norm(*phi[l], 0), go[l]->norm(*phi[l], 0));
    scalar(l, "norm1", ro[l]->norm(*phi[l], 1), go[l]->norm(*phi[l], 1));
    scalar(l, "norm2", ro[l]->norm(*phi[l], 2), go[l]->norm(*phi[l], 2));
    scalar(l, "dotProduct", ro[l]->dotProduct(*phi[l], *rhs[l]), go[l]->dotProduct(*phi[l], *rhs[l]));
    {
      Pair* x = mk(g, phi[l]);
      ro[l]->incr(x->r, *rhs[l], -0.37);
      go[l]->incr(x->g, *rhs[l], -0.37);
      report(l, "incr", validDiff(x->r, x->g));
      ro[l]->axby(x->r, *phi[l], *rhs[l], 0.3, -1.7);
      go[l]->axby(x->g, *phi[l], *rhs[l], 0.3, -1.7);
      report(l, "axby", validDiff(x->r, x->g));
      ro[l]->scale(x->r, 1.9);
      go[l]->scale(x->g, 1.9);
      report(l, "scale", validDiff(x->r, x->g));
      delete x;
    }
  }
  // Multigrid depths below level 0: relax, residual, restrictResidual and
  // prolongIncrement, each depth against the next.
  std::vector<MGLevelOp<LDF>*> rm, gm;
  rm.push_back(ro[0]);
  gm.push_back(go[0]);
  for (int d = 1;; ++d) {
    MGLevelOp<LDF>* r = refFactory->MGnewOp(P.domains[0], d, true);
    MGLevelOp<LDF>* gg = gpuFactory->MGnewOp(P.domains[0], d, true);
    if ((r == nullptr) != (gg == nullptr)) {
      std::printf("{\"error\": \"multigrid depth %d exists on one side only\"}\n", d);
      return 3;
    }
    if (!r) break;
    rm.push_back(r);
    gm.push_back(gg);
  }
  std::vector<LDF*> mphi(rm.size()), mrhs(rm.size());
  mphi[0] = phi[0];
  mrhs[0] = rhs[0];
  for (size_t d = 1; d < rm.size(); ++d) {
    mphi[d] = new LDF;
    mrhs[d] = new LDF;
    rm[d - 1]->createCoarser(*mphi[d], *mphi[d - 1], true);
    rm[d - 1]->createCoarser(*mrhs[d], *mrhs[d - 1], false);
    seededField(*mphi[d], P.dxs[0] * (1 << d), prob.bumps, 17u + (unsigned)d);
    seededField(*mrhs[d], P.dxs[0] * (1 << d), prob.bumps, 91u + (unsigned)d);
  }
  for (size_t d = 1; d < rm.size(); ++d) {
    const int lev = -(int)d;
    const DisjointBoxLayout& g = mphi[d]->disjointBoxLayout();
    {
      Pair *ph = mk(g, mphi[d]), *out = mk(g, nullptr);
      rm[d]->residual(out->r, ph->r, *mrhs[d], true);
      gm[d]->residual(out->g, ph->g, *mrhs[d], true);
      report(lev, "residual_homog", validDiff(out->r, out->g));
      delete ph;
      delete out;
    }
    {
      Pair* ph = mk(g, mphi[d]);
      rm[d]->relax(ph->r, *mrhs[d], 2);
      gm[d]->relax(ph->g, *mrhs[d], 2);
      report(lev, "relax2", validDiff(ph->r, ph->g));
      delete ph;
    }
    {
      Pair* ph = mk(g, mphi[d]);
      rm[d]->preCond(ph->r, *mrhs[d]);
      gm[d]->preCond(ph->g, *mrhs[d]);
      report(lev, "preCond", validDiff(ph->r, ph->g));
      delete ph;
    }
    {  // restriction from depth d - 1 into depth d, prolongation back
      const DisjointBoxLayout& gf = mphi[d - 1]->disjointBoxLayout();
      Pair *ph = mk(gf, mphi[d - 1]), *rc = mk(g, nullptr);
      rm[d - 1]->restrictResidual(rc->r, ph->r, *mrhs[d - 1]);
      gm[d - 1]->restrictResidual(rc->g, ph->g, *mrhs[d - 1]);
      report(lev + 1, "restrictResidual", validDiff(rc->r, rc->g));
      Pair* pf = mk(gf, mphi[d - 1]);
      rm[d - 1]->prolongIncrement(pf->r, *mphi[d]);
      gm[d - 1]->prolongIncrement(pf->g, *mphi[d]);
      report(lev + 1, "prolongIncrement", validDiff(pf->r, pf->g));
      delete ph;
      delete rc;
      delete pf;
    }
    scalar(lev, "norm2", rm[d]->norm(*mphi[d], 2), gm[d]->norm(*mphi[d], 2));
    scalar(lev, "dotProduct", rm[d]->dotProduct(*mphi[d], *mrhs[d]), gm[d]->dotProduct(*mphi[d], *mrhs[d]));
  }
  json += "]}";
  std::printf("%s\n", json.c_str());
  return 0;
}

// The bottom solver the multigrid solves are given: the reference's
// BiCGStabSolver, or with relaxbottom=1 its RelaxSolver (the AMRINS
// projection's bottom solver, CCProjector.cpp:1056-1058), defaults kept.
static LinearSolver<LDF>* newBottom() {
  if (argd("relaxbottom", 0) != 0) {
    RelaxSolver<LDF>* r = new RelaxSolver<LDF>;
    r->m_verbosity = 0;
    return r;
  }
  BiCGStabSolver<LDF>* b = new BiCGStabSolver<LDF>;
  b->m_verbosity = 0;
  return b;
}

// The reference's own AMRMultiGrid (or, with fas=1, its AMRFASMultiGrid in
// V-cycle mode), unmodified, defined once with the reference's factory and
// once with the GPU factory (cmg_chombo's AMRLevelOpFactory, whose operators
// run on the device one call at a time): both solves print exit status,
// iteration count, residual history and phi deviation as one JSON line.
// AMRFASMultiGrid calls no inspector, so its history is the final composite
// residual alone.
static int amrmgCheck(OracleProblem& P, Vector<int>& rr) {
  const bool fas = argd("fas", 0) != 0;
  const int nlev = P.nlev, lmax = P.finest;
  const int pre = (int)argd("pre", 4), post = (int)argd("post", 4), bottom = (int)argd("bottom", 4);
  const int iters = (int)argd("iters", 100);
  const Real eps = argd("eps", 1e-10), hang = argd("hang", 1e-10);
  RefCountedPtr<AMRLevelOpFactory<LDF> > refFactory;
  if (P.opType == 0) {
    AMRPoissonOpFactory* f = new AMRPoissonOpFactory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    refFactory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    refFactory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  }
  cmg_chombo::GpuAMRPoissonOpFactory gpf;
  cmg_chombo::GpuVCAMRPoissonOp2Factory gvf;
  AMRLevelOpFactory<LDF>* gpuFactory = &gpf;
  if (P.opType == 0)
    gpf.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
  else {
    gvf.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    gpuFactory = &gvf;
  }
  Vector<LDF*> phiG(nlev);
  for (int l = 0; l < nlev; ++l) {
    phiG[l] = new LDF(P.grids[l], 1, IntVect::Unit);
    for (DataIterator dit = P.grids[l].dataIterator(); dit.ok(); ++dit) phiG[l]->operator[](dit()).setVal(0.0);
  }
  ResidualRecorder* recs[2];
  int exitS[2], itersDone[2];
  for (int side = 0; side < 2; ++side) {
    LinearSolver<LDF>* bottomSolver = newBottom();
    AMRFASMultiGrid<LDF>* fmg = fas ? new AMRFASMultiGrid<LDF> : nullptr;
    AMRMultiGrid<LDF>* mg = fas ? fmg : new AMRMultiGrid<LDF>;
    mg->define(P.domains[0], side == 0 ? *refFactory : *gpuFactory, bottomSolver, nlev);
    mg->setSolverParameters(pre, post, bottom, 1, iters, eps, hang, 1e-30);
    mg->m_verbosity = 0;
    RefCountedPtr<AMRMultiGridInspector<LDF> > insp(new ResidualRecorder);
    mg->addInspector(insp);
    mg->solve(side == 0 ? P.phi : phiG, P.rhs, lmax, 0, true);
    recs[side] = static_cast<ResidualRecorder*>(&(*insp));
    recs[side]->norms.push_back(mg->computeAMRResidual(side == 0 ? P.phi : phiG, P.rhs, lmax, 0));
    itersDone[side] = fas ? fmg->m_iter : (int)recs[side]->norms.size() - 1;
    exitS[side] = mg->m_exitStatus;
    insp.neverDelete();
    delete mg;
    delete bottomSolver;
  }
  const bool sameLen = recs[0]->norms.size() == recs[1]->norms.size();
  bool histExact = sameLen;
  double maxHist = 0;
  if (sameLen)
    for (size_t i = 0; i < recs[0]->norms.size(); ++i) {
      histExact = histExact && recs[0]->norms[i] == recs[1]->norms[i];
      maxHist = std::max(maxHist, std::fabs(recs[0]->norms[i] - recs[1]->norms[i]) / recs[0]->norms[0]);
    }
  long ndiff = 0;
  std::string perLevel;
  for (int l = 0; l < nlev; ++l) {
    const long d = validDiff(*P.phi[l], *phiG[l]).ndiff;
    ndiff += d;
    perLevel += (l ? ", " : "") + std::to_string(d);
  }
  std::printf("{\"amrmg\": 1, \"fas\": %d, \"levels\": %d, \"cpu_exit\": %d, \"gpu_exit\": %d, \"cpu_iters\": %d, \"gpu_iters\": %d, "
              "\"same_history_length\": %s, \"history_exact\": %s, \"history_dev\": %.3e, \"phi_ndiff\": %ld, "
              "\"phi_rel_dev\": %.3e, \"phi_ndiff_per_level\": [%s]}\n",
              fas ? 1 : 0, nlev, exitS[0], exitS[1], itersDone[0], itersDone[1],
              sameLen ? "true" : "false", histExact ? "true" : "false", maxHist, ndiff, phiDeviation(P, phiG),
              perLevel.c_str());
  delete recs[0];
  delete recs[1];
  return 0;
}

// An inhomogeneous Dirichlet boundary condition (value 1 on every face,
// ghost = 2*1 - inside) handed to the GPU factory: define() must stop with
// MayDay::Error, which aborts this program.
static void oneValue(Real*, int*, Side::LoHiSide*, Real* a_values) { a_values[0] = 1.; }
static void inhomDirichletBC(FArrayBox& a_state, const Box& a_valid, const ProblemDomain& a_domain, Real a_dx,
                             bool a_homogeneous) {
  for (int i = 0; i < CH_SPACEDIM; ++i)
    for (SideIterator sit; sit.ok(); ++sit) {
      Box g = adjCellBox(a_valid, i, sit(), 1);
      if (a_domain.domainBox().contains(g)) continue;
      DiriBC(a_state, a_valid, a_dx, a_homogeneous, oneValue, i, sit(), 1);
    }
}

int main(int argc, char** argv) {
  for (int a = 1; a < argc; ++a) {
    const char* eq = std::strchr(argv[a], '=');
    if (eq) g_args[std::string(argv[a], eq - argv[a])] = std::string(eq + 1);
  }
  if (g_args.count("bc")) setFaceBC(g_args["bc"]);
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
  if (argd("ops", 0) != 0) return opsCheck(P, rr);
  if (argd("amrmg", 0) != 0) return amrmgCheck(P, rr);
  if (argd("badbc", 0) != 0) {
    cmg_chombo::GpuAMRPoissonOpFactory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &inhomDirichletBC, P.alpha, P.beta);
    std::printf("{\"inhomogeneous_accepted\": true}\n");
    return 0;
  }
  if (argd("bcprobe", 0) != 0) {  // the face types the GPU factory reads off the problem's BC function
    cmg_chombo::GpuAMRPoissonOpFactory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    const int* t = f.description().bc;
    std::printf("{\"bc_types\": [%d, %d, %d, %d, %d, %d]}\n", t[0], t[1], t[2], t[3], t[4], t[5]);
    return 0;
  }

  // Reference: CPU AMRMultiGrid.
  RefCountedPtr<AMRLevelOpFactory<LDF> > factory;
  if (P.opType == 0) {
    AMRPoissonOpFactory* f = new AMRPoissonOpFactory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  } else {
    VCAMRPoissonOp2Factory* f = new VCAMRPoissonOp2Factory;
    f->define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
    factory = RefCountedPtr<AMRLevelOpFactory<LDF> >(f);
  }
  LinearSolver<LDF>* bottomSolver = newBottom();
  AMRMultiGrid<LDF> cpu;
  cpu.define(P.domains[0], *factory, bottomSolver, nlev);
  cpu.setSolverParameters(pre, post, bottom, 1, iters, eps, hang, 1e-30);
  cpu.m_verbosity = 0;
  RefCountedPtr<AMRMultiGridInspector<LDF> > insp(new ResidualRecorder);
  cpu.addInspector(insp);
  cpu.solve(P.phi, P.rhs, lmax, 0, true);
  ResidualRecorder* rec = static_cast<ResidualRecorder*>(&(*insp));
  rec->norms.push_back(cpu.computeAMRResidual(P.phi, P.rhs, lmax, 0));

  // The same calls on the GPU drop-in.
  cmg_chombo::GpuAMRMultiGrid gpu;
  LinearSolver<LDF>* gpuBottomPtr = newBottom();
  LinearSolver<LDF>& gpuBottom = *gpuBottomPtr;
  if (P.opType == 0) {
    cmg_chombo::GpuAMRPoissonOpFactory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.beta);
    gpu.define(P.domains[0], f, &gpuBottom, nlev);
  } else {
    cmg_chombo::GpuVCAMRPoissonOp2Factory f;
    f.define(P.domains[0], P.grids, rr, P.dxs[0], &domainBC, P.alpha, P.aCoef, P.beta, P.bCoef);
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
