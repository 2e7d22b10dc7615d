// Chombo-side drop-in for the GPU solve: the API of AMRMultiGrid<LevelData<
// FArrayBox>> with AMRPoissonOpFactory / VCAMRPoissonOp2Factory, implemented
// over the C ABI of cmg.h (libcmg.so).  A Chombo 3.2 program switches
//
//     AMRPoissonOpFactory f;     f.define(domain, grids, refRatios, dx, bc, alpha, beta);
//     AMRMultiGrid<LevelData<FArrayBox> > s;
//     s.define(domain, f, &bottomSolver, numLevels);
//     s.setSolverParameters(pre, post, bottom, numMG, iterMax, eps, hang, normThresh);
//     s.solve(phi, rhs, numLevels - 1, 0);
//
// to the same calls on cmg_chombo::GpuAMRPoissonOpFactory and
// cmg_chombo::GpuAMRMultiGrid (or GpuVCAMRPoissonOp2Factory), with the same
// arguments, and gets the same valid-cell phi (FP64, identical operation
// order; see the parity tests), the same m_exitStatus and the same residual
// history.  The header needs the Chombo headers (serial, 3D, double) and is
// compiled inside the Chombo program; link with -lcmg.
//
// Scope, each checked with MayDay::Error like the reference's own checks:
//   - refinement ratio 2 between all levels, non-periodic domain, serial
//     (every box local), one component;
//   - homogeneous Dirichlet boundary conditions on the domain faces (the
//     examples' ParseBC with value 0, order 1): the BCHolder argument is kept
//     for signature compatibility and is not called;
//   - the bottom solver must be a BiCGStabSolver (its device restatement runs
//     with the reference's default parameters);
//   - solve over all levels: l_base = 0 and l_max = numLevels - 1.
// Only valid cells of phi are written; ghost cells are left as they were.
//
// The variable-coefficient example's solve path has its drop-in too:
// MultilevelLinearOp<FArrayBox> + BiCGStabSolver<Vector<LevelData<FArrayBox>*>>
// become cmg_chombo::GpuMultilevelLinearOp + GpuMultilevelBiCGStabSolver with
// the same members and calls (define with the GPU factory, solve(phi, rhs)).
#ifndef CMG_CHOMBO_H
#define CMG_CHOMBO_H

#include <vector>

#include "BCFunc.H"
#include "BiCGStabSolver.H"
#include "DisjointBoxLayout.H"
#include "FArrayBox.H"
#include "FluxBox.H"
#include "LevelData.H"
#include "LinearSolver.H"
#include "MayDay.H"
#include "ProblemDomain.H"
#include "RealVect.H"
#include "RefCountedPtr.H"
#include "cmg.h"

namespace cmg_chombo {

typedef LevelData<FArrayBox> LDF;

// What an operator factory conveys to the solver.
struct GpuOpDescription {
  ProblemDomain coarseDomain;
  Vector<DisjointBoxLayout> grids;
  Vector<int> refRatios;
  Real coarsedx = 0, alpha = 0, beta = 1;
  int vc = 0;
  Vector<RefCountedPtr<LDF> > aCoef;
  Vector<RefCountedPtr<LevelData<FluxBox> > > bCoef;
  bool defined = false;
};

// AMRPoissonOpFactory::define (AMRElliptic/AMRPoissonOp.H:535-541).
class GpuAMRPoissonOpFactory {
 public:
  void define(const ProblemDomain& a_coarseDomain, const Vector<DisjointBoxLayout>& a_grids,
              const Vector<int>& a_refRatios, const Real& a_coarsedx, BCHolder /*a_bc*/, Real a_alpha = 0.0,
              Real a_beta = 1.0) {
    m_d = GpuOpDescription();
    m_d.coarseDomain = a_coarseDomain;
    m_d.grids = a_grids;
    m_d.refRatios = a_refRatios;
    m_d.coarsedx = a_coarsedx;
    m_d.alpha = a_alpha;
    m_d.beta = a_beta;
    m_d.vc = 0;
    m_d.defined = true;
  }
  const GpuOpDescription& description() const { return m_d; }

 private:
  GpuOpDescription m_d;
};

// VCAMRPoissonOp2Factory::define (AMRElliptic/VCAMRPoissonOp2.H:278-286).
// The coefficients are read when GpuAMRMultiGrid::define runs (the reference
// computes its relaxation coefficient from them at the same point).
class GpuVCAMRPoissonOp2Factory {
 public:
  void define(const ProblemDomain& a_coarseDomain, const Vector<DisjointBoxLayout>& a_grids,
              const Vector<int>& a_refRatios, const Real& a_coarsedx, BCHolder /*a_bc*/, const Real& a_alpha,
              Vector<RefCountedPtr<LDF> >& a_aCoef, const Real& a_beta,
              Vector<RefCountedPtr<LevelData<FluxBox> > >& a_bCoef) {
    m_d = GpuOpDescription();
    m_d.coarseDomain = a_coarseDomain;
    m_d.grids = a_grids;
    m_d.refRatios = a_refRatios;
    m_d.coarsedx = a_coarsedx;
    m_d.alpha = a_alpha;
    m_d.beta = a_beta;
    m_d.vc = 1;
    m_d.aCoef = a_aCoef;
    m_d.bCoef = a_bCoef;
    m_d.defined = true;
  }
  const GpuOpDescription& description() const { return m_d; }

 private:
  GpuOpDescription m_d;
};

// AMRMultiGrid<LevelData<FArrayBox>> (AMRElliptic/AMRMultiGrid.H:301-470):
// define, setSolverParameters, solve, computeAMRResidual, m_exitStatus.
// The device hierarchy behind the drop-ins: the factory's description turned
// into a cmg_hierarchy, and LevelData valid cells moved to and from it.
class GpuHierarchy {
 public:
  GpuHierarchy() {}
  ~GpuHierarchy() { clear(); }
  GpuHierarchy(const GpuHierarchy&) = delete;
  GpuHierarchy& operator=(const GpuHierarchy&) = delete;
  void clear() {
    if (m_h) cmg_hierarchy_destroy(m_h);
    m_h = nullptr;
    m_nlev = 0;
  }
  cmg_hierarchy* handle() const { return m_h; }
  int numLevels() const { return m_nlev; }

  static void check(int rc) {
    if (rc != CMG_OK) MayDay::Error(cmg_last_error());
  }

  int64_t cells(int l) const {
    int64_t n = 0;
    check(cmg_num_cells(m_h, l, &n));
    return n;
  }

  // Valid cells of every box in layout order, x fastest (the C ABI's order).
  void pack(const LDF& a_ld, int l, std::vector<double>& out) const {
    out.clear();
    const DisjointBoxLayout& dbl = m_d.grids[l];
    for (DataIterator dit = a_ld.dataIterator(); dit.ok(); ++dit) {
      const Box& b = dbl[dit()];
      const FArrayBox& f = a_ld[dit];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
          for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) out.push_back(f(IntVect(i, j, k), 0));
    }
  }

  void unpack(const std::vector<double>& in, int l, LDF& a_ld) const {
    size_t p = 0;
    const DisjointBoxLayout& dbl = m_d.grids[l];
    for (DataIterator dit = a_ld.dataIterator(); dit.ok(); ++dit) {
      const Box& b = dbl[dit()];
      FArrayBox& f = a_ld[dit];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
          for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) f(IntVect(i, j, k), 0) = in[p++];
    }
  }

  void setLevels(const Vector<LDF*>& a_data, bool phi) const {
    std::vector<double> buf;
    for (int l = 0; l < m_nlev; ++l) {
      pack(*a_data[l], l, buf);
      check(phi ? cmg_set_phi(m_h, l, buf.data(), 0) : cmg_set_rhs(m_h, l, buf.data(), 0));
    }
  }

  void getPhi(Vector<LDF*>& a_phi) const {
    std::vector<double> buf;
    for (int l = 0; l < m_nlev; ++l) {
      buf.resize(cells(l));
      check(cmg_get_phi(m_h, l, buf.data(), 0));
      unpack(buf, l, *a_phi[l]);
    }
  }

  void defineFrom(const ProblemDomain& a_coarseDomain, const GpuOpDescription& d, int a_numLevels) {
    clear();
    if (!d.defined) MayDay::Error("cmg_chombo: factory not defined");
    if (a_numLevels < 1 || a_numLevels > d.grids.size()) MayDay::Error("cmg_chombo: bad number of levels");
    for (int l = 0; l + 1 < a_numLevels; ++l)
      if (d.refRatios[l] != 2) MayDay::Error("cmg_chombo: refinement ratio 2 only");
    for (int dir = 0; dir < SpaceDim; ++dir)
      if (a_coarseDomain.isPeriodic(dir)) MayDay::Error("cmg_chombo: periodic domains are not supported");
    m_d = d;
    m_nlev = a_numLevels;
    std::vector<int> counts;
    std::vector<cmg_box> boxes;
    for (int l = 0; l < m_nlev; ++l) {
      const DisjointBoxLayout& dbl = d.grids[l];
      int n = 0;
      for (LayoutIterator lit = dbl.layoutIterator(); lit.ok(); ++lit, ++n) {
        const Box& b = dbl[lit()];
        cmg_box c;
        for (int dir = 0; dir < 3; ++dir) {
          c.lo[dir] = b.smallEnd(dir);
          c.hi[dir] = b.bigEnd(dir);
        }
        boxes.push_back(c);
      }
      counts.push_back(n);
    }
    const Box& db = a_coarseDomain.domainBox();
    int lo[3], hi[3];
    for (int dir = 0; dir < 3; ++dir) {
      lo[dir] = db.smallEnd(dir);
      hi[dir] = db.bigEnd(dir);
    }
    check(cmg_hierarchy_create(lo, hi, d.coarsedx, m_nlev, counts.data(), boxes.data(), d.vc, d.alpha, d.beta,
                               &m_h));
    if (d.vc) {
      std::vector<double> buf;
      for (int l = 0; l < m_nlev; ++l) {
        pack(*d.aCoef[l], l, buf);
        check(cmg_set_acoef(m_h, l, buf.data(), 0));
        for (int dir = 0; dir < 3; ++dir) {
          buf.clear();
          const LevelData<FluxBox>& bc = *d.bCoef[l];
          for (DataIterator dit = bc.dataIterator(); dit.ok(); ++dit) {
            const Box fb = surroundingNodes(d.grids[l][dit()], dir);
            const FArrayBox& f = bc[dit][dir];
            for (int k = fb.smallEnd(2); k <= fb.bigEnd(2); ++k)
              for (int j = fb.smallEnd(1); j <= fb.bigEnd(1); ++j)
                for (int i = fb.smallEnd(0); i <= fb.bigEnd(0); ++i) buf.push_back(f(IntVect(i, j, k), 0));
          }
          check(cmg_set_bcoef(m_h, l, dir, buf.data(), 0));
        }
      }
      check(cmg_finalize_coefficients(m_h));
    }
  }

 protected:
  cmg_hierarchy* m_h = nullptr;
  int m_nlev = 0;
  GpuOpDescription m_d;
};

class GpuAMRMultiGrid : private GpuHierarchy {
  friend class GpuBackwardEuler;
  friend class GpuAMRTGA;

 public:
  int m_exitStatus = 0;
  int m_verbosity = 0;

  GpuAMRMultiGrid() {}

  void define(const ProblemDomain& a_coarseDomain, GpuAMRPoissonOpFactory& a_factory, LinearSolver<LDF>* a_bottom,
              int a_numLevels) {
    defineWith(a_coarseDomain, a_factory.description(), a_bottom, a_numLevels);
  }
  void define(const ProblemDomain& a_coarseDomain, GpuVCAMRPoissonOp2Factory& a_factory, LinearSolver<LDF>* a_bottom,
              int a_numLevels) {
    defineWith(a_coarseDomain, a_factory.description(), a_bottom, a_numLevels);
  }

  // AMRMultiGrid::setSolverParameters (AMRMultiGrid.H:451-458, 527-546).
  void setSolverParameters(const int& a_pre, const int& a_post, const int& a_bottom, const int& a_numMG,
                           const int& a_iterMax, const Real& a_eps, const Real& a_hang, const Real& a_normThresh) {
    m_p.pre = a_pre;
    m_p.post = a_post;
    m_p.bottom = a_bottom;
    m_p.num_mg = a_numMG;
    m_p.iter_max = a_iterMax;
    m_p.eps = a_eps;
    m_p.hang = a_hang;
    m_p.norm_thresh = a_normThresh;
  }

  // AMRMultiGrid::solve (AMRMultiGrid.H:894-1124) on the device.
  void solve(Vector<LDF*>& a_phi, const Vector<LDF*>& a_rhs, int l_max, int l_base, bool a_zeroPhi = true,
             bool /*forceHomogeneous*/ = false) {
    checkRange(l_max, l_base);
    setLevels(a_rhs, false);
    if (!a_zeroPhi) setLevels(a_phi, true);
    m_history.assign(m_p.iter_max + 2, 0.0);
    int st = 0, it = 0, hl = 0;
    check(cmg_solve(m_h, &m_p, a_zeroPhi ? 1 : 0, &st, &it, m_history.data(), (int)m_history.size(), &hl));
    m_history.resize(hl);
    m_exitStatus = st;
    m_iterations = it;
    getPhi(a_phi);
  }

  // AMRMultiGrid::computeAMRResidual(phi, rhs, l_max, l_base) (AMRMultiGrid.H:738-750):
  // the composite max-norm residual of the given phi and rhs.
  Real computeAMRResidual(Vector<LDF*>& a_phi, const Vector<LDF*>& a_rhs, int l_max, int l_base) {
    checkRange(l_max, l_base);
    setLevels(a_rhs, false);
    setLevels(a_phi, true);
    double r = 0;
    check(cmg_residual_norm(m_h, &r));
    return r;
  }

  // Composite max-norm residual at the start of every iteration of the last
  // solve, then the final one (what an AMRMultiGridInspector would record).
  const std::vector<double>& residualHistory() const { return m_history; }
  int iterations() const { return m_iterations; }

  void clear() { GpuHierarchy::clear(); }

 private:
  cmg_solve_params m_p = {4, 4, 4, 1, 100, 5, 1e-10, 1e-10, 1e-30};
  std::vector<double> m_history;
  int m_iterations = 0;

  void checkRange(int l_max, int l_base) const {
    if (!m_h) MayDay::Error("GpuAMRMultiGrid: solve before define");
    if (l_base != 0 || l_max != m_nlev - 1)
      MayDay::Error("GpuAMRMultiGrid: only l_base = 0, l_max = numLevels - 1 is supported");
  }

  void defineWith(const ProblemDomain& a_coarseDomain, const GpuOpDescription& d, LinearSolver<LDF>* a_bottom,
                  int a_numLevels) {
    if (a_bottom && !dynamic_cast<BiCGStabSolver<LDF>*>(a_bottom))
      MayDay::Error("GpuAMRMultiGrid: the device solve uses BiCGStab as its bottom solver");
    defineFrom(a_coarseDomain, d, a_numLevels);
  }
};

// The reference's heat solvers over the GPU solve: BackwardEuler
// (AMRElliptic/BackwardEuler.cpp) and AMRTGA<LevelData<FArrayBox>>
// (AMRElliptic/AMRTGA.H), same constructor and oneStep arguments, built on a
// GpuAMRMultiGrid (its solver parameters are the solves').  Each oneStep
// moves phiOld and the source to the device, runs the step there
// (cmg_backward_euler / cmg_tga) and returns phiNew; lbase 0 and
// lmax = numLevels - 1 only.
class GpuBackwardEuler {
 public:
  template <class Factory>
  GpuBackwardEuler(const RefCountedPtr<GpuAMRMultiGrid>& a_solver, const Factory& /*a_opFact*/,
                   const ProblemDomain& /*a_level0Domain*/, const Vector<int>& /*a_refRat*/, int /*a_numLevels*/ = -1,
                   int /*a_verbosity*/ = 3)
      : m_solver(a_solver) {}

  void oneStep(Vector<LDF*>& a_phiNew, Vector<LDF*>& a_phiOld, Vector<LDF*>& a_source, const Real& a_dt,
               int a_lbase, int a_lmax, bool a_zeroPhi = true) {
    GpuAMRMultiGrid& s = *m_solver;
    s.checkRange(a_lmax, a_lbase);
    s.setLevels(a_phiOld, true);
    s.setLevels(a_source, false);
    int st = 0, it = 0;
    GpuHierarchy::check(cmg_backward_euler(s.m_h, &s.m_p, a_dt, 1, a_zeroPhi ? 1 : 0, &st, &it));
    s.m_exitStatus = st;
    s.m_iterations = it;
    s.getPhi(a_phiNew);
  }

 private:
  RefCountedPtr<GpuAMRMultiGrid> m_solver;
};

class GpuAMRTGA {
 public:
  template <class Factory>
  GpuAMRTGA(const RefCountedPtr<GpuAMRMultiGrid>& a_solver, const Factory& /*a_factory*/,
            const ProblemDomain& /*a_level0Domain*/, const Vector<int>& /*a_refRat*/, int /*a_numLevels*/ = -1,
            int /*a_verbosity*/ = 0)
      : m_solver(a_solver) {}

  void oneStep(Vector<LDF*>& a_phiNew, Vector<LDF*>& a_phiOld, Vector<LDF*>& a_source, const Real& a_dt,
               int a_lbase, int a_lmax, Real /*a_timeOld*/ = 0) {
    GpuAMRMultiGrid& s = *m_solver;
    s.checkRange(a_lmax, a_lbase);
    s.setLevels(a_phiOld, true);
    s.setLevels(a_source, false);
    int st[2] = {0, 0}, it[2] = {0, 0};
    GpuHierarchy::check(cmg_tga(s.m_h, &s.m_p, a_dt, 1, st, it));
    s.m_exitStatus = st[1];
    s.m_iterations = it[1];
    s.getPhi(a_phiNew);
  }

 private:
  RefCountedPtr<GpuAMRMultiGrid> m_solver;
};

// MultilevelLinearOp<FArrayBox> (AMRElliptic/MultilevelLinearOp.H) for the
// GPU factories: the multilevel operator with the AMR multigrid
// preconditioner, as the variable-coefficient example defines it
// (VCPoissonSolve.cpp:148-167).  Supported: lBase 0, the multigrid
// preconditioner at full depth (m_preCondSolverDepth -1).
class GpuMultilevelLinearOp : public GpuHierarchy {
 public:
  bool m_use_multigrid_preconditioner = true;
  int m_num_mg_iterations = 1;
  int m_num_mg_smooth = 4;
  int m_preCondSolverDepth = -1;

  void define(const Vector<DisjointBoxLayout>& a_vectGrids, const Vector<int>& /*a_refRatios*/,
              const Vector<ProblemDomain>& a_domains, const Vector<RealVect>& /*a_vectDx*/,
              GpuAMRPoissonOpFactory& a_factory, int a_lBase) {
    defineWith(a_vectGrids, a_domains, a_factory.description(), a_lBase);
  }
  void define(const Vector<DisjointBoxLayout>& a_vectGrids, const Vector<int>& /*a_refRatios*/,
              const Vector<ProblemDomain>& a_domains, const Vector<RealVect>& /*a_vectDx*/,
              GpuVCAMRPoissonOp2Factory& a_factory, int a_lBase) {
    defineWith(a_vectGrids, a_domains, a_factory.description(), a_lBase);
  }

 private:
  void defineWith(const Vector<DisjointBoxLayout>& a_vectGrids, const Vector<ProblemDomain>& a_domains,
                  const GpuOpDescription& d, int a_lBase) {
    if (a_lBase != 0) MayDay::Error("GpuMultilevelLinearOp: only lBase = 0 is supported");
    if (a_domains.size() < 1) MayDay::Error("GpuMultilevelLinearOp: no domains");
    defineFrom(a_domains[0], d, a_vectGrids.size());
  }
};

// BiCGStabSolver<Vector<LevelData<FArrayBox>*>> over GpuMultilevelLinearOp
// (BiCGStabSolver.H:199-515 with MultilevelLinearOp's vector operations):
// the same members and solve(phi, rhs), phi being the initial guess.  The
// max norm (m_normType 0, what the example sets) is supported; no
// convergence metric (m_convergenceMetric <= 0).
class GpuMultilevelBiCGStabSolver {
 public:
  bool m_homogeneous = false;
  int m_imax = 80;
  int m_verbosity = 3;
  Real m_eps = 1.0E-6;
  Real m_reps = 1.0E-12;
  Real m_convergenceMetric = -1.0;
  Real m_hang = 1E-8;
  int m_exitStatus = -1;
  int m_iter = -1;
  Real m_residual = -1e300;
  Real m_initial_residual = -1e300;
  Real m_small = 1.0E-30;
  int m_numRestarts = 5;
  int m_normType = 2;

  void define(GpuMultilevelLinearOp* a_operator, bool a_homogeneous) {
    m_op = a_operator;
    m_homogeneous = a_homogeneous;
  }

  void solve(Vector<LDF*>& a_phi, const Vector<LDF*>& a_rhs) {
    if (!m_op || !m_op->handle()) MayDay::Error("GpuMultilevelBiCGStabSolver: solve before define");
    if (m_normType != 0) MayDay::Error("GpuMultilevelBiCGStabSolver: only the max norm (m_normType 0) is supported");
    if (m_convergenceMetric > 0) MayDay::Error("GpuMultilevelBiCGStabSolver: convergence metrics are not supported");
    if (!m_op->m_use_multigrid_preconditioner || m_op->m_preCondSolverDepth >= 0)
      MayDay::Error("GpuMultilevelBiCGStabSolver: only the full-depth multigrid preconditioner is supported");
    if (a_phi.size() != m_op->numLevels() || a_rhs.size() != m_op->numLevels())
      MayDay::Error("GpuMultilevelBiCGStabSolver: level count differs from the operator's");
    m_op->setLevels(a_rhs, false);
    m_op->setLevels(a_phi, true);
    cmg_mlsolve_params p = {m_op->m_num_mg_iterations, m_op->m_num_mg_smooth, m_imax, m_numRestarts,
                            m_eps, m_reps, m_hang, m_small};
    m_history.assign(m_imax + 1, 0.0);
    int hl = 0;
    double r0 = 0, rf = 0;
    GpuHierarchy::check(cmg_solve_multilevel_bicgstab(m_op->handle(), &p, 0, &m_exitStatus, &m_iter, &r0, &rf,
                                                      m_history.data(), (int)m_history.size(), &hl));
    m_history.resize(hl);
    m_initial_residual = r0;
    m_residual = rf;
    m_op->getPhi(a_phi);
  }

  // Residual norm after every iteration of the last solve.
  const std::vector<double>& residualHistory() const { return m_history; }

 private:
  GpuMultilevelLinearOp* m_op = nullptr;
  std::vector<double> m_history;
};

// FineInterp (AMRTools/FineInterp.H:35-245) on the device: define() with the
// fine layout, one component, refinement ratio 2 and the fine problem domain;
// interpToFine / pwcinterpToFine send the coarse data's valid cells, run
// cmg_fine_interp_run and write every valid cell of the fine data, with the
// reference's default PCInterp boundary limiting.  The device plan is built
// on the first call for a coarse layout and kept while that layout is the
// same object.  Only properly nested levels are accepted (the reference then
// reads nothing but coarse data), so a_averageFromDest, whose averages the
// coarse copy overwrites on such levels (FineInterp.cpp:124-148), changes
// nothing.
class GpuFineInterp {
 public:
  GpuFineInterp() {}
  GpuFineInterp(const DisjointBoxLayout& a_fine_domain, const int& a_numcomps, const int& a_ref_ratio,
                const ProblemDomain& a_fine_problem_domain) {
    define(a_fine_domain, a_numcomps, a_ref_ratio, a_fine_problem_domain);
  }
  GpuFineInterp(const DisjointBoxLayout& a_fine_domain, const int& a_numcomps, const int& a_ref_ratio,
                const Box& a_fine_problem_domain) {
    define(a_fine_domain, a_numcomps, a_ref_ratio, ProblemDomain(a_fine_problem_domain));
  }
  ~GpuFineInterp() { clear(); }
  GpuFineInterp(const GpuFineInterp&) = delete;
  GpuFineInterp& operator=(const GpuFineInterp&) = delete;

  void define(const DisjointBoxLayout& a_fine_domain, const int& a_numcomps, const int& a_ref_ratio,
              const ProblemDomain& a_fine_problem_domain) {
    if (a_numcomps != 1) MayDay::Error("cmg_chombo: GpuFineInterp takes one component");
    if (a_ref_ratio != 2) MayDay::Error("cmg_chombo: refinement ratio 2 only");
    for (int dir = 0; dir < SpaceDim; ++dir)
      if (a_fine_problem_domain.isPeriodic(dir)) MayDay::Error("cmg_chombo: periodic domains are not supported");
    clear();
    m_fine = a_fine_domain;
    m_domain = a_fine_problem_domain.domainBox();
    m_defined = true;
  }
  void define(const DisjointBoxLayout& a_fine_domain, const int& a_numcomps, const int& a_ref_ratio,
              const Box& a_fine_problem_domain) {
    define(a_fine_domain, a_numcomps, a_ref_ratio, ProblemDomain(a_fine_problem_domain));
  }
  bool isDefined() const { return m_defined; }

  void interpToFine(LevelData<FArrayBox>& a_fine_data, const LevelData<FArrayBox>& a_coarse_data,
                    bool a_averageFromDest = false) {
    run(a_fine_data, a_coarse_data, false);
  }
  void pwcinterpToFine(LevelData<FArrayBox>& a_fine_data, const LevelData<FArrayBox>& a_coarse_data,
                       bool a_averageFromDest = false) {
    run(a_fine_data, a_coarse_data, true);
  }

 private:
  static void boxesOf(const DisjointBoxLayout& g, std::vector<cmg_box>& out) {
    out.clear();
    for (LayoutIterator lit = g.layoutIterator(); lit.ok(); ++lit) {
      const Box& b = g[lit];
      cmg_box c;
      for (int d = 0; d < 3; ++d) {
        c.lo[d] = b.smallEnd(d);
        c.hi[d] = b.bigEnd(d);
      }
      out.push_back(c);
    }
  }
  void clear() {
    if (m_h) cmg_fine_interp_destroy(m_h);
    m_h = nullptr;
  }
  void run(LevelData<FArrayBox>& a_fine, const LevelData<FArrayBox>& a_coarse, bool pwc) {
    if (!m_defined) MayDay::Error("cmg_chombo: GpuFineInterp not defined");
    if (a_coarse.nComp() != 1 || a_fine.nComp() != 1) MayDay::Error("cmg_chombo: GpuFineInterp takes one component");
    const DisjointBoxLayout& cg = a_coarse.disjointBoxLayout();
    if (!m_h || !(cg == m_coarse)) {
      clear();
      std::vector<cmg_box> fb, cb;
      boxesOf(m_fine, fb);
      boxesOf(cg, cb);
      const int lo[3] = {m_domain.smallEnd(0), m_domain.smallEnd(1), m_domain.smallEnd(2)};
      const int hi[3] = {m_domain.bigEnd(0), m_domain.bigEnd(1), m_domain.bigEnd(2)};
      GpuHierarchy::check(cmg_fine_interp_create(lo, hi, (int)fb.size(), fb.data(), (int)cb.size(), cb.data(), &m_h));
      m_coarse = cg;
    }
    std::vector<double> in, out;
    for (DataIterator dit = a_coarse.dataIterator(); dit.ok(); ++dit) {
      const Box& b = cg[dit()];
      const FArrayBox& f = a_coarse[dit];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
          for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) in.push_back(f(IntVect(i, j, k), 0));
    }
    out.resize(m_fine.numCells());
    GpuHierarchy::check(cmg_fine_interp_run(m_h, in.data(), out.data(), 0, pwc ? 1 : 0));
    size_t p = 0;
    for (DataIterator dit = a_fine.dataIterator(); dit.ok(); ++dit) {
      const Box& b = m_fine[dit()];
      FArrayBox& f = a_fine[dit];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
          for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) f(IntVect(i, j, k), 0) = out[p++];
    }
  }
  bool m_defined = false;
  DisjointBoxLayout m_fine, m_coarse;
  Box m_domain;
  cmg_fine_interp* m_h = nullptr;
};

}  // namespace cmg_chombo

#endif
