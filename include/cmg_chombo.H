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
//   - homogeneous Dirichlet or homogeneous Neumann boundary conditions, one
//     type per domain face (the examples' ParseBC with value 0, order 1; the
//     AMRINS projection's walls and outflow).  The factories' define()
//     probes the BCHolder: on a two-cell slab along each of the six domain
//     faces it calls the BC (inhomogeneous) and requires every face ghost to
//     be minus the cell inside it (Dirichlet) or equal to it (Neumann); any
//     other condition (a non-zero value, a higher-order stencil) is rejected
//     there;
//   - the bottom solver is a BiCGStabSolver or a RelaxSolver; its public
//     parameters (m_imax, m_numRestarts, m_normType 2 or 0, m_eps of the
//     RelaxSolver, m_hang, m_small) are read when each solve starts;
//   - solve over all levels: l_base = 0 and l_max = numLevels - 1.
// Only valid cells of phi are written; ghost cells are left as they were.
//
// The factories are also AMRLevelOpFactory<LevelData<FArrayBox>>s: the
// reference's own, unmodified AMRMultiGrid (or MultiGrid, BiCGStabSolver or
// any other caller of the operator interface) can be defined with them and
// drives GpuAMRPoissonOp objects one virtual at a time.  Each call moves its
// LevelData arguments to the device and back (the cmg_op_* entry points),
// which is correct but slow; GpuAMRMultiGrid, whose hierarchy stays on the
// device for the whole solve, is the fast path.
//
// The variable-coefficient example's solve path has its drop-in too:
// MultilevelLinearOp<FArrayBox> + BiCGStabSolver<Vector<LevelData<FArrayBox>*>>
// become cmg_chombo::GpuMultilevelLinearOp + GpuMultilevelBiCGStabSolver with
// the same members and calls (define with the GPU factory, solve(phi, rhs)).
#ifndef CMG_CHOMBO_H
#define CMG_CHOMBO_H

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "AMRMultiGrid.H"
#include "BCFunc.H"
#include "BiCGStabSolver.H"
#include "DisjointBoxLayout.H"
#include "FArrayBox.H"
#include "FluxBox.H"
#include "LevelData.H"
#include "LinearSolver.H"
#include "LevelDataOps.H"
#include "MayDay.H"
#include "ProblemDomain.H"
#include "RealVect.H"
#include "RelaxSolver.H"
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
  int bc[6] = {0, 0, 0, 0, 0, 0};  // per domain face: CMG_BC_DIRICHLET, _NEUMANN or _PERIODIC (probeBoundary)
  Vector<RefCountedPtr<LDF> > aCoef;
  Vector<RefCountedPtr<LevelData<FluxBox> > > bCoef;
  bool defined = false;
};

// The boundary type of every domain face of a_bc, which the device solve
// supports when it is homogeneous Dirichlet (ghost = 2*0 - inside,
// BCFunc.cpp:294-354 with value 0, order 1) or homogeneous Neumann (ghost =
// inside, BCFunc.cpp:217-236 with value 0), as the drivers' ParseBC and the
// AMRINS projection's pressure BC function set them: on a slab two cells deep
// along each domain face the BC is called inhomogeneous on distinct cell
// values, and every ghost across that face must be minus the cell next to it
// (Dirichlet) or equal to it (Neumann).  Anything else stops with
// MayDay::Error.
inline void probeBoundary(BCHolder a_bc, const ProblemDomain& a_domain, Real a_dx, int a_types[6]) {
  const Box& d = a_domain.domainBox();
  for (int dir = 0; dir < SpaceDim; ++dir)
    for (SideIterator sit; sit.ok(); ++sit) {
      if (a_domain.isPeriodic(dir)) {
        // The operators never apply a BC across a periodic face: its ghost
        // cells are exchanged from the domain's periodic image.
        a_types[2 * dir + (sit() == Side::Hi ? 1 : 0)] = CMG_BC_PERIODIC;
        continue;
      }
      Box valid = d;
      const int w = std::min(2, d.size(dir));
      if (sit() == Side::Lo)
        valid.setBig(dir, d.smallEnd(dir) + w - 1);
      else
        valid.setSmall(dir, d.bigEnd(dir) - w + 1);
      FArrayBox fab(grow(valid, 1), 1);
      fab.setVal(1.0e30);
      for (BoxIterator bit(valid); bit.ok(); ++bit) {
        const IntVect& iv = bit();
        fab(iv, 0) = 1.0 + 0.25 * iv[0] + 7.0 * iv[1] + 53.0 * iv[2];
      }
      a_bc(fab, valid, a_domain, a_dx, false);
      const Box ghost = adjCellBox(valid, dir, sit(), 1);
      const IntVect in = (sit() == Side::Lo ? 1 : -1) * BASISV(dir);
      bool diri = true, neu = true;
      for (BoxIterator bit(ghost); bit.ok(); ++bit) {
        diri = diri && fab(bit(), 0) == -fab(bit() + in, 0);
        neu = neu && fab(bit(), 0) == fab(bit() + in, 0);
      }
      if (!diri && !neu)
        MayDay::Error("cmg_chombo: the device operators support homogeneous Dirichlet (ghost = -inside) and "
                      "homogeneous Neumann (ghost = inside) boundary conditions only; this BCHolder sets "
                      "something else on a domain face");
      a_types[2 * dir + (sit() == Side::Hi ? 1 : 0)] = diri ? CMG_BC_DIRICHLET : CMG_BC_NEUMANN;
    }
}

inline bool sameBoxes(const DisjointBoxLayout& a, const DisjointBoxLayout& b) {
  if (a.size() != b.size()) return false;
  LayoutIterator ia = a.layoutIterator(), ib = b.layoutIterator();
  for (; ia.ok() && ib.ok(); ++ia, ++ib)
    if (a[ia()] != b[ib()]) return false;
  return true;
}

class GpuHierarchy;

// AMRPoissonOp / VCAMRPoissonOp2 (AMRElliptic/AMRPoissonOp.H:35-510,
// VCAMRPoissonOp2.H:25-249) as an AMRLevelOp over the device hierarchy of
// its factory: one AMR level (lev >= 0) or one multigrid depth below level 0
// (lev = -depth).  Every operator method sends its LevelData arguments (in
// the ghosted format of cmg.h: each FAB grown by one cell) to the matching
// cmg_op_* call and writes the valid cells of its outputs back; ghost cells
// of the caller's data are left as they were.  Container methods (create,
// createCoarser, createCoarsened, assign, assignLocal, setToZero,
// buildCopier) are the reference's LevelData operations.
class GpuAMRPoissonOp : public AMRLevelOp<LDF> {
 public:
  GpuAMRPoissonOp(std::shared_ptr<GpuHierarchy> a_h, int a_lev, const DisjointBoxLayout& a_grids, Real a_dx,
                  const DisjointBoxLayout* a_finerCoarsened)
      : m_sh(a_h), m_lev(a_lev), m_grids(a_grids), m_dx(a_dx) {
    if (a_finerCoarsened) {
      m_finerCoarsened = *a_finerCoarsened;
      m_hasFiner = true;
    }
  }
  virtual ~GpuAMRPoissonOp() {}

  int level() const { return m_lev; }

  // ---------------------------------------------------------------- LinearOp
  virtual void residual(LDF& a_lhs, const LDF& a_phi, const LDF& a_rhs, bool a_homogeneous = false) {
    in(a_phi, m_a);
    in(a_rhs, m_b);
    out0(m_o);
    check(cmg_op_residual(h(), m_lev, m_o.data(), m_a.data(), m_b.data(), a_homogeneous ? 1 : 0));
    outValid(m_o, a_lhs);
  }
  virtual void preCond(LDF& a_cor, const LDF& a_residual) {
    in(a_cor, m_a);
    in(a_residual, m_b);
    check(cmg_op_precond(h(), m_lev, m_a.data(), m_b.data()));
    outValid(m_a, a_cor);
  }
  virtual void applyOp(LDF& a_lhs, const LDF& a_phi, bool a_homogeneous = false) {
    in(a_phi, m_a);
    out0(m_o);
    check(cmg_op_apply(h(), m_lev, m_o.data(), m_a.data(), a_homogeneous ? 1 : 0));
    outValid(m_o, a_lhs);
  }
  // LevelDataOps::create / assign / assignLocal / setToZero (LevelDataOps.H).
  virtual void create(LDF& a_lhs, const LDF& a_rhs) {
    a_lhs.define(a_rhs.disjointBoxLayout(), a_rhs.nComp(), a_rhs.ghostVect());
  }
  virtual void assign(LDF& a_lhs, const LDF& a_rhs) { a_rhs.copyTo(a_rhs.interval(), a_lhs, a_lhs.interval()); }
  virtual void assignLocal(LDF& a_lhs, const LDF& a_rhs) {
    for (DataIterator dit = a_lhs.dataIterator(); dit.ok(); ++dit) a_lhs[dit].copy(a_rhs[dit]);
  }
  // BLAS-1 on data of this level runs on the device; FASMultiGrid also hands
  // the finest operator data of other depths (FASMultiGrid.H cycle), which
  // goes to the reference's own LevelDataOps, as in the reference.
  virtual Real dotProduct(const LDF& a_1, const LDF& a_2) {
    if (!mine(a_1)) return m_ops.dotProduct(a_1, a_2);
    in(a_1, m_a);
    in(a_2, m_b);
    double r = 0;
    check(cmg_op_dot(h(), m_lev, m_a.data(), m_b.data(), &r));
    return r;
  }
  virtual void incr(LDF& a_lhs, const LDF& a_x, Real a_scale) {
    if (!mine(a_lhs)) return m_ops.incr(a_lhs, a_x, a_scale);
    in(a_lhs, m_o);
    in(a_x, m_a);
    check(cmg_op_incr(h(), m_lev, m_o.data(), m_a.data(), a_scale));
    outValid(m_o, a_lhs);
  }
  virtual void axby(LDF& a_lhs, const LDF& a_x, const LDF& a_y, Real a_a, Real a_b) {
    if (!mine(a_lhs)) return m_ops.axby(a_lhs, a_x, a_y, a_a, a_b);
    in(a_x, m_a);
    in(a_y, m_b);
    out0(m_o);
    check(cmg_op_axby(h(), m_lev, m_o.data(), m_a.data(), m_b.data(), a_a, a_b));
    outValid(m_o, a_lhs);
  }
  virtual void scale(LDF& a_lhs, const Real& a_scale) {
    if (!mine(a_lhs)) return m_ops.scale(a_lhs, a_scale);
    in(a_lhs, m_o);
    check(cmg_op_scale(h(), m_lev, m_o.data(), a_scale));
    outValid(m_o, a_lhs);
  }
  virtual Real norm(const LDF& a_x, int a_ord) {
    if (!mine(a_x)) return CH_XD::norm(a_x, a_x.interval(), a_ord);
    in(a_x, m_a);
    double r = 0;
    check(cmg_op_norm(h(), m_lev, m_a.data(), a_ord, &r));
    return r;
  }
  virtual void setToZero(LDF& a_lhs) {
    for (DataIterator dit = a_lhs.dataIterator(); dit.ok(); ++dit) a_lhs[dit].setVal(0.0);
  }
  virtual Real dx() const { return m_dx; }

  // ---------------------------------------------------------------- MGLevelOp
  virtual void createCoarser(LDF& a_coarse, const LDF& a_fine, bool /*a_ghosted*/) {
    DisjointBoxLayout dbl;
    coarsen(dbl, a_fine.disjointBoxLayout(), 2);
    a_coarse.define(dbl, a_fine.nComp(), a_fine.ghostVect());
  }
  virtual void relax(LDF& a_correction, const LDF& a_residual, int a_iterations) {
    in(a_correction, m_a);
    in(a_residual, m_b);
    check(cmg_op_relax(h(), m_lev, m_a.data(), m_b.data(), a_iterations));
    outValid(m_a, a_correction);
  }
  // AMRPoissonOp::relaxNF (AMRPoissonOp.cpp:586-596): the inhomogeneous
  // coarse-fine ghosts from a_phiCoarse, then relax.
  virtual void relaxNF(LDF& a_phi, const LDF* a_phiCoarse, const LDF& a_rhs, int a_iterations) {
    if (a_phiCoarse != NULL) coarseFineInterp(a_phi, *a_phiCoarse);
    relax(a_phi, a_rhs, a_iterations);
  }
  // AMRPoissonOp::residualNF (AMRPoissonOp.cpp:238-254): homogeneous
  // coarse-fine ghosts, or inhomogeneous ones from a_phiCoarse, then
  // residualI (which keeps the coarse-fine ghosts a_phi holds).
  virtual void residualNF(LDF& a_lhs, LDF& a_phi, const LDF* a_phiCoarse, const LDF& a_rhs,
                          bool a_homogeneous = false) {
    if (!a_homogeneous && a_phiCoarse != NULL) coarseFineInterp(a_phi, *a_phiCoarse);
    residual(a_lhs, a_phi, a_rhs, a_homogeneous);
  }
  virtual void restrictResidual(LDF& a_resCoarse, LDF& a_phiFine, const LDF& a_rhsFine) {
    in(a_phiFine, m_a);
    in(a_rhsFine, m_b);
    packGhosted(a_resCoarse, m_o);
    check(cmg_op_restrict_residual(h(), m_lev, m_o.data(), m_a.data(), m_b.data()));
    unpackValid(m_o, a_resCoarse);
  }
  virtual void prolongIncrement(LDF& a_phiThisLevel, const LDF& a_correctCoarse) {
    in(a_phiThisLevel, m_a);
    packGhosted(a_correctCoarse, m_b);
    check(cmg_op_prolong_increment(h(), m_lev, m_a.data(), m_b.data()));
    outValid(m_a, a_phiThisLevel);
  }

  // ---------------------------------------------------------------- AMRLevelOp
  virtual int refToCoarser() { return 2; }
  virtual void AMRResidual(LDF& a_residual, const LDF& a_phiFine, const LDF& a_phi, const LDF& a_phiCoarse,
                           const LDF& a_rhs, bool, AMRLevelOp<LDF>*) {
    amrOp(1, a_residual, &a_phiFine, a_phi, &a_phiCoarse, &a_rhs);
  }
  virtual void AMRResidualNF(LDF& a_residual, const LDF& a_phi, const LDF& a_phiCoarse, const LDF& a_rhs, bool) {
    amrOp(2, a_residual, nullptr, a_phi, &a_phiCoarse, &a_rhs);
  }
  virtual void AMRResidualNC(LDF& a_residual, const LDF& a_phiFine, const LDF& a_phi, const LDF& a_rhs, bool,
                             AMRLevelOp<LDF>*) {
    amrOp(1, a_residual, &a_phiFine, a_phi, nullptr, &a_rhs);
  }
  virtual void AMROperator(LDF& a_LofPhi, const LDF& a_phiFine, const LDF& a_phi, const LDF& a_phiCoarse, bool,
                           AMRLevelOp<LDF>*) {
    amrOp(0, a_LofPhi, &a_phiFine, a_phi, &a_phiCoarse, nullptr);
  }
  virtual void AMROperatorNF(LDF& a_LofPhi, const LDF& a_phi, const LDF& a_phiCoarse, bool) {
    amrOp(0, a_LofPhi, nullptr, a_phi, &a_phiCoarse, nullptr);
  }
  virtual void AMROperatorNC(LDF& a_LofPhi, const LDF& a_phiFine, const LDF& a_phi, bool, AMRLevelOp<LDF>*) {
    amrOp(0, a_LofPhi, &a_phiFine, a_phi, nullptr, nullptr);
  }
  virtual void AMRRestrict(LDF& a_resCoarse, const LDF& a_residual, const LDF& a_correction,
                           const LDF& a_coarseCorrection, bool a_skip_res) {
    LDF scratch;
    AMRRestrictS(a_resCoarse, a_residual, a_correction, a_coarseCorrection, scratch, a_skip_res);
  }
  virtual void AMRRestrictS(LDF& a_resCoarse, const LDF& a_residual, const LDF& a_correction,
                            const LDF& a_coarseCorrection, LDF& /*scratch*/, bool a_skip_res = false) {
    in(a_residual, m_a);
    if (!a_skip_res) {
      in(a_correction, m_b);
      packGhosted(a_coarseCorrection, m_c);
    }
    int64_t n = 0;
    check(cmg_op_coarsened_size(h(), m_lev, &n));
    m_o.resize(n);
    check(cmg_op_amr_restrict(h(), m_lev, m_o.data(), m_a.data(), a_skip_res ? nullptr : m_b.data(),
                              a_skip_res ? nullptr : m_c.data()));
    unpackValid(m_o, a_resCoarse);
  }
  virtual void AMRProlong(LDF& a_correction, const LDF& a_coarseCorrection) {
    in(a_correction, m_a);
    packGhosted(a_coarseCorrection, m_b);
    check(cmg_op_amr_prolong(h(), m_lev, m_a.data(), m_b.data()));
    outValid(m_a, a_correction);
  }
  virtual void AMRProlongS(LDF& a_correction, const LDF& a_coarseCorrection, LDF& /*a_temp*/,
                           const Copier& /*a_copier*/) {
    AMRProlong(a_correction, a_coarseCorrection);
  }
  virtual void AMRUpdateResidual(LDF& a_residual, const LDF& a_correction, const LDF& a_coarseCorrection) {
    in(a_residual, m_o);
    in(a_correction, m_a);
    packGhosted(a_coarseCorrection, m_b);
    check(cmg_op_amr_update_residual(h(), m_lev, m_o.data(), m_a.data(), m_b.data()));
    outValid(m_o, a_residual);
  }
  virtual void createCoarsened(LDF& a_lhs, const LDF& a_rhs, const int& a_refRat) {
    DisjointBoxLayout dbl;
    coarsen(dbl, a_rhs.disjointBoxLayout(), a_refRat);
    a_lhs.define(dbl, a_rhs.nComp(), a_rhs.ghostVect());
  }
  // AMRPoissonOp::buildCopier (AMRPoissonOp.cpp:474-483).
  virtual void buildCopier(Copier& a_copier, const LDF& a_lhs, const LDF& a_rhs) {
    a_copier.define(a_rhs.disjointBoxLayout(), a_lhs.disjointBoxLayout(), a_lhs.ghostVect());
  }
  // The coarsened-fine residual of the next finer level onto this level
  // (AMRMultiGrid::AMRVCycle) runs on the device; any other copy is the
  // reference's copyTo with the given copier.
  virtual void assignCopier(LDF& a_lhs, const LDF& a_rhs, const Copier& a_copier) {
    if (m_hasFiner && sameBoxes(a_lhs.disjointBoxLayout(), m_grids) &&
        sameBoxes(a_rhs.disjointBoxLayout(), m_finerCoarsened)) {
      in(a_lhs, m_o);
      packGhosted(a_rhs, m_a);
      check(cmg_op_assign_coarsened(h(), m_lev + 1, m_o.data(), m_a.data()));
      outValid(m_o, a_lhs);
    } else {
      a_rhs.copyTo(a_rhs.interval(), a_lhs, a_lhs.interval(), a_copier);
    }
  }
  virtual void zeroCovered(LDF& a_lhs, LDF& a_rhs, const Copier& a_copier) {
    setToZero(a_rhs);
    if (m_hasFiner && sameBoxes(a_lhs.disjointBoxLayout(), m_grids) &&
        sameBoxes(a_rhs.disjointBoxLayout(), m_finerCoarsened)) {
      in(a_lhs, m_o);
      check(cmg_op_zero_covered(h(), m_lev, m_o.data()));
      outValid(m_o, a_lhs);
    } else {
      a_rhs.copyTo(a_rhs.interval(), a_lhs, a_lhs.interval(), a_copier);
    }
  }
  virtual Real localMaxNorm(const LDF& a_phi) { return norm(a_phi, 0); }

  // QuadCFInterp::coarseFineInterp of this level (AMRPoissonOp's
  // m_interpWithCoarser): the coarse-fine ghosts of a_phi from a_phiCoarse.
  void coarseFineInterp(LDF& a_phi, const LDF& a_phiCoarse) {
    if (m_lev < 1) MayDay::Error("cmg_chombo: coarseFineInterp on a level without a coarser level");
    in(a_phi, m_a);
    packGhosted(a_phiCoarse, m_b);
    check(cmg_op_cf_interp(h(), m_lev, m_a.data(), m_b.data()));
    unpackGrown(m_a, a_phi);
  }

 private:
  std::shared_ptr<GpuHierarchy> m_sh;
  int m_lev;
  DisjointBoxLayout m_grids, m_finerCoarsened;
  bool m_hasFiner = false;
  Real m_dx;
  std::vector<double> m_a, m_b, m_c, m_o;

  LevelDataOps<FArrayBox> m_ops;

  bool mine(const LDF& a_ld) const { return sameBoxes(a_ld.disjointBoxLayout(), m_grids); }
  cmg_hierarchy* h() const;
  static void check(int rc) {
    if (rc != CMG_OK) MayDay::Error(cmg_last_error());
  }

 public:
  // Every FAB of a_ld grown by one cell (zero where the FAB has no ghost
  // layer), box after box in layout order: the cmg.h ghosted format.
  static void packGhosted(const LDF& a_ld, std::vector<double>& a_out) {
    a_out.clear();
    const DisjointBoxLayout& dbl = a_ld.disjointBoxLayout();
    for (DataIterator dit = a_ld.dataIterator(); dit.ok(); ++dit) {
      const Box g = grow(dbl[dit()], 1);
      const FArrayBox& f = a_ld[dit];
      const size_t base = a_out.size();
      a_out.resize(base + g.numPts());
      double* o = a_out.data() + base;
      if (f.box() == g) {
        std::memcpy(o, f.dataPtr(0), g.numPts() * sizeof(double));
        continue;
      }
      const Box fb = f.box();
      size_t q = 0;
      for (int k = g.smallEnd(2); k <= g.bigEnd(2); ++k)
        for (int j = g.smallEnd(1); j <= g.bigEnd(1); ++j)
          for (int i = g.smallEnd(0); i <= g.bigEnd(0); ++i, ++q) {
            const IntVect iv(i, j, k);
            o[q] = fb.contains(iv) ? f(iv, 0) : 0.0;
          }
    }
  }
  // Every cell of a ghosted array that a_ld's FABs hold (valid and ghost).
  static void unpackGrown(const std::vector<double>& a_in, LDF& a_ld) {
    const DisjointBoxLayout& dbl = a_ld.disjointBoxLayout();
    size_t base = 0;
    for (DataIterator dit = a_ld.dataIterator(); dit.ok(); ++dit) {
      const Box g = grow(dbl[dit()], 1);
      FArrayBox& f = a_ld[dit];
      const Box r = g & f.box();
      for (BoxIterator bit(r); bit.ok(); ++bit) {
        const IntVect& iv = bit();
        f(iv, 0) = a_in[base + (iv[0] - g.smallEnd(0)) +
                        (size_t)g.size(0) * ((iv[1] - g.smallEnd(1)) + (size_t)g.size(1) * (iv[2] - g.smallEnd(2)))];
      }
      base += g.numPts();
    }
  }
  // The valid cells of a ghosted array into a_ld.
  static void unpackValid(const std::vector<double>& a_in, LDF& a_ld) {
    const DisjointBoxLayout& dbl = a_ld.disjointBoxLayout();
    size_t base = 0;
    for (DataIterator dit = a_ld.dataIterator(); dit.ok(); ++dit) {
      const Box& b = dbl[dit()];
      const Box g = grow(b, 1);
      const int gx = g.size(0), gy = g.size(1), nx = b.size(0);
      FArrayBox& f = a_ld[dit];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j) {
          const double* src = a_in.data() + base + 1 + (size_t)gx * ((j - g.smallEnd(1)) + (size_t)gy * (k - g.smallEnd(2)));
          std::memcpy(&f(IntVect(b.smallEnd(0), j, k), 0), src, nx * sizeof(double));
        }
      base += g.numPts();
    }
  }

 private:
  void in(const LDF& a_ld, std::vector<double>& a_buf) const {
    if (!sameBoxes(a_ld.disjointBoxLayout(), m_grids))
      MayDay::Error("cmg_chombo: LevelData on another layout than the operator's level");
    packGhosted(a_ld, a_buf);
  }
  void out0(std::vector<double>& a_buf) const {
    int64_t n = 0;
    check(cmg_op_size(h(), m_lev, &n));
    a_buf.assign(n, 0.0);
  }
  void outValid(const std::vector<double>& a_buf, LDF& a_ld) const {
    if (!sameBoxes(a_ld.disjointBoxLayout(), m_grids))
      MayDay::Error("cmg_chombo: LevelData on another layout than the operator's level");
    unpackValid(a_buf, a_ld);
  }
  void amrOp(int a_form, LDF& a_out, const LDF* a_phiFine, const LDF& a_phi, const LDF* a_phiCoarse,
             const LDF* a_rhs) {
    const bool fine = a_phiFine && a_phiFine->isDefined();
    const bool coarse = a_phiCoarse && a_phiCoarse->isDefined() && m_lev > 0;
    in(a_phi, m_a);
    if (a_rhs) in(*a_rhs, m_b);
    if (fine) packGhosted(*a_phiFine, m_c);
    if (coarse) packGhosted(*a_phiCoarse, m_d);
    out0(m_o);
    check(cmg_op_amr_operator(h(), m_lev, a_form, m_o.data(), fine ? m_c.data() : nullptr, m_a.data(),
                              coarse ? m_d.data() : nullptr, a_rhs ? m_b.data() : nullptr));
    outValid(m_o, a_out);
    // The reference fills the ghost cells of its const phi argument
    // (coarse-fine, exchange, boundary) and later operators that apply the
    // stencil without a coarse-fine fill (AMROperatorNC, residual with
    // inhomogeneous boundaries) read them: keep them the same here.
    unpackGrown(m_a, const_cast<LDF&>(a_phi));
  }
  std::vector<double> m_d;
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
    if (a_coarseDomain.isPeriodic() && a_numLevels > 1)
      MayDay::Error("cmg_chombo: periodic domains are supported for one-level hierarchies only");
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
    check(cmg_hierarchy_create_bc(lo, hi, d.coarsedx, m_nlev, counts.data(), boxes.data(), d.vc, d.alpha, d.beta,
                                  d.bc, &m_h));
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

inline cmg_hierarchy* GpuAMRPoissonOp::h() const { return m_sh->handle(); }

// What AMRPoissonOpFactory and VCAMRPoissonOp2Factory share as
// AMRLevelOpFactory<LevelData<FArrayBox>> (AMRElliptic/AMRMultiGrid.H:233-251,
// MultiGrid.H:295-320): AMRnewOp for each AMR level's domain, MGnewOp for the
// multigrid depths below level 0 (AMRPoissonOp.cpp:1923-1989: depth d exists
// while level 0's boxes coarsen by 2^(d+1)), refToFiner.  The device
// hierarchy behind the operators is built at the first AMRnewOp / MGnewOp
// after define() (the VC coefficients are read then, as the reference's
// factory computes its relaxation coefficient when it makes an operator) and
// shared by every operator made from it.  MGnewOp below a refined level
// returns NULL: with refinement ratio 2 between AMR levels the reference's
// AMRMultiGrid never runs those depths (AMRMultiGrid::init sets their
// MultiGrid depth to 0).
class GpuOpFactoryBase : public AMRLevelOpFactory<LDF> {
 public:
  virtual ~GpuOpFactoryBase() {}
  const GpuOpDescription& description() const { return m_d; }

  virtual AMRLevelOp<LDF>* AMRnewOp(const ProblemDomain& a_indexSpace) {
    const int l = levelOf(a_indexSpace);
    std::shared_ptr<GpuHierarchy> sh = shared();
    if (l >= sh->numLevels()) MayDay::Error("cmg_chombo: AMRnewOp for a level without boxes");
    return newOp(sh, l);
  }
  virtual MGLevelOp<LDF>* MGnewOp(const ProblemDomain& a_fineIndexSpace, int a_depth, bool /*a_homoOnly*/ = true) {
    const int l = levelOf(a_fineIndexSpace);
    std::shared_ptr<GpuHierarchy> sh = shared();
    if (l >= sh->numLevels()) MayDay::Error("cmg_chombo: MGnewOp for a level without boxes");
    if (a_depth == 0) return newOp(sh, l);
    int depths = 0;
    GpuHierarchy::check(cmg_op_num_mg_depths(sh->handle(), &depths));
    if (l > 0 || a_depth > depths) return nullptr;
    return newOp(sh, -a_depth);
  }
  virtual int refToFiner(const ProblemDomain& a_indexSpace) const {
    const int l = levelOf(a_indexSpace);
    return l < m_d.refRatios.size() ? m_d.refRatios[l] : 2;
  }

 protected:
  GpuOpDescription m_d;
  BCHolder m_bc;
  std::shared_ptr<GpuHierarchy> m_shared;

  void redefine(const GpuOpDescription& a_d, BCHolder a_bc) {
    m_d = a_d;
    m_bc = a_bc;
    m_shared.reset();
    probeBoundary(a_bc, a_d.coarseDomain, a_d.coarsedx, m_d.bc);
  }
  int levelOf(const ProblemDomain& a_domain) const {
    if (!m_d.defined) MayDay::Error("cmg_chombo: factory not defined");
    ProblemDomain dom = m_d.coarseDomain;
    for (int l = 0; l < m_d.grids.size(); ++l) {
      if (dom.domainBox() == a_domain.domainBox()) return l;
      if (l < m_d.refRatios.size()) dom.refine(m_d.refRatios[l]);
    }
    MayDay::Error("cmg_chombo: operator requested for a domain of no level");
    return -1;
  }
  std::shared_ptr<GpuHierarchy> shared();
  GpuAMRPoissonOp* newOp(const std::shared_ptr<GpuHierarchy>& a_sh, int a_lev) const;
};

// AMRPoissonOpFactory::define (AMRElliptic/AMRPoissonOp.H:535-541).
class GpuAMRPoissonOpFactory : public GpuOpFactoryBase {
 public:
  void define(const ProblemDomain& a_coarseDomain, const Vector<DisjointBoxLayout>& a_grids,
              const Vector<int>& a_refRatios, const Real& a_coarsedx, BCHolder a_bc, Real a_alpha = 0.0,
              Real a_beta = 1.0) {
    GpuOpDescription d;
    d.coarseDomain = a_coarseDomain;
    d.grids = a_grids;
    d.refRatios = a_refRatios;
    d.coarsedx = a_coarsedx;
    d.alpha = a_alpha;
    d.beta = a_beta;
    d.vc = 0;
    d.defined = true;
    redefine(d, a_bc);
  }
};

// VCAMRPoissonOp2Factory::define (AMRElliptic/VCAMRPoissonOp2.H:278-286).
// The coefficients are read when the device hierarchy is built (the first
// operator made, or GpuAMRMultiGrid::define).
class GpuVCAMRPoissonOp2Factory : public GpuOpFactoryBase {
 public:
  void define(const ProblemDomain& a_coarseDomain, const Vector<DisjointBoxLayout>& a_grids,
              const Vector<int>& a_refRatios, const Real& a_coarsedx, BCHolder a_bc, const Real& a_alpha,
              Vector<RefCountedPtr<LDF> >& a_aCoef, const Real& a_beta,
              Vector<RefCountedPtr<LevelData<FluxBox> > >& a_bCoef) {
    GpuOpDescription d;
    d.coarseDomain = a_coarseDomain;
    d.grids = a_grids;
    d.refRatios = a_refRatios;
    d.coarsedx = a_coarsedx;
    d.alpha = a_alpha;
    d.beta = a_beta;
    d.vc = 1;
    d.aCoef = a_aCoef;
    d.bCoef = a_bCoef;
    d.defined = true;
    redefine(d, a_bc);
  }
};

inline std::shared_ptr<GpuHierarchy> GpuOpFactoryBase::shared() {
  if (!m_shared) {
    int nlev = 0;
    while (nlev < m_d.grids.size() && m_d.grids[nlev].size() > 0) ++nlev;
    std::shared_ptr<GpuHierarchy> sh(new GpuHierarchy);
    sh->defineFrom(m_d.coarseDomain, m_d, nlev);
    m_shared = sh;
  }
  return m_shared;
}

inline GpuAMRPoissonOp* GpuOpFactoryBase::newOp(const std::shared_ptr<GpuHierarchy>& a_sh, int a_lev) const {
  if (a_lev >= 0) {
    Real dx = m_d.coarsedx;
    for (int l = 0; l < a_lev; ++l) dx /= m_d.refRatios[l];
    DisjointBoxLayout finer;
    const bool hasFiner = a_lev + 1 < a_sh->numLevels();
    if (hasFiner) coarsen(finer, m_d.grids[a_lev + 1], 2);
    return new GpuAMRPoissonOp(a_sh, a_lev, m_d.grids[a_lev], dx, hasFiner ? &finer : nullptr);
  }
  const int coarsening = 1 << (-a_lev);
  DisjointBoxLayout g;
  coarsen(g, m_d.grids[0], coarsening);
  return new GpuAMRPoissonOp(a_sh, a_lev, g, m_d.coarsedx * coarsening, nullptr);
}

// AMRMultiGrid<LevelData<FArrayBox>> (AMRElliptic/AMRMultiGrid.H:301-470) on
// the device: define, setSolverParameters, solve, computeAMRResidual, and the
// reference's public solver members with its defaults (AMRMultiGrid.H:
// 599-622): eps 1e-6, hang 1e-15, normThresh 1e-30, imin 5, iterMax 20,
// iterMin -1, pre = post = bottom = 2, one V-cycle per level.
class GpuAMRMultiGrid : private GpuHierarchy {
  friend class GpuBackwardEuler;
  friend class GpuAMRTGA;

 public:
  Real m_eps = 1e-6, m_hang = 1e-15, m_normThresh = 1e-30;
  int m_imin = 5, m_iterMax = 20, m_iterMin = -1, m_verbosity = 3, m_exitStatus = -1;
  int m_pre = 2, m_post = 2, m_bottom = 2, m_numMG = 1;

  GpuAMRMultiGrid() {}

  void define(const ProblemDomain& a_coarseDomain, GpuOpFactoryBase& a_factory, LinearSolver<LDF>* a_bottom,
              int a_numLevels) {
    defineWith(a_coarseDomain, a_factory.description(), a_bottom, a_numLevels);
  }

  // AMRMultiGrid::setSolverParameters (AMRMultiGrid.H:451-458, 527-546).
  void setSolverParameters(const int& a_pre, const int& a_post, const int& a_bottom, const int& a_numMG,
                           const int& a_iterMax, const Real& a_eps, const Real& a_hang, const Real& a_normThresh) {
    m_pre = a_pre;
    m_post = a_post;
    m_bottom = a_bottom;
    m_numMG = a_numMG;
    m_iterMax = a_iterMax;
    m_eps = a_eps;
    m_hang = a_hang;
    m_normThresh = a_normThresh;
  }

  // AMRMultiGrid::solve (AMRMultiGrid.H:894-1124) on the device.
  // forceHomogeneous changes nothing: the boundary values are zero either way.
  // A residual norm that turns NaN or infinite ends the solve (the C ABI's
  // CMG_EDIVERGED); phi and m_exitStatus are set as for any other end, with a
  // warning, as the reference's loop also stops on a NaN norm.
  void solve(Vector<LDF*>& a_phi, const Vector<LDF*>& a_rhs, int l_max, int l_base, bool a_zeroPhi = true,
             bool /*forceHomogeneous*/ = false) {
    checkRange(l_max, l_base);
    setLevels(a_rhs, false);
    if (!a_zeroPhi) setLevels(a_phi, true);
    const cmg_solve_params p = params();
    applyBottom();
    m_history.assign(std::max(p.iter_max, p.iter_min) + 2, 0.0);
    int st = 0, it = 0, hl = 0;
    const int rc = cmg_solve(m_h, &p, a_zeroPhi ? 1 : 0, &st, &it, m_history.data(), (int)m_history.size(), &hl);
    if (rc == CMG_EDIVERGED)
      MayDay::Warning(cmg_last_error());
    else
      check(rc);
    m_history.resize(std::min<size_t>(hl, m_history.size()));
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
  std::vector<double> m_history;
  int m_iterations = 0;

  cmg_solve_params params() const {
    cmg_solve_params p;
    p.pre = m_pre;
    p.post = m_post;
    p.bottom = m_bottom;
    p.num_mg = m_numMG;
    p.iter_max = m_iterMax;
    p.imin = m_imin;
    p.eps = m_eps;
    p.hang = m_hang;
    p.norm_thresh = m_normThresh;
    p.iter_min = m_iterMin;
    return p;
  }

  void checkRange(int l_max, int l_base) const {
    if (!m_h) MayDay::Error("GpuAMRMultiGrid: solve before define");
    if (l_base != 0 || l_max != m_nlev - 1)
      MayDay::Error("GpuAMRMultiGrid: only l_base = 0, l_max = numLevels - 1 is supported");
  }

  void defineWith(const ProblemDomain& a_coarseDomain, const GpuOpDescription& d, LinearSolver<LDF>* a_bottom,
                  int a_numLevels) {
    if (a_bottom && !dynamic_cast<BiCGStabSolver<LDF>*>(a_bottom) && !dynamic_cast<RelaxSolver<LDF>*>(a_bottom))
      MayDay::Error("GpuAMRMultiGrid: the device bottom solver is a BiCGStabSolver or a RelaxSolver");
    m_bottomSolver = a_bottom;
    defineFrom(a_coarseDomain, d, a_numLevels);
  }

  // The bottom solver's public parameters, read when a solve starts (as the
  // reference reads them inside its solve).
  void applyBottom() {
    cmg_bottom_params b = {CMG_BOTTOM_BICGSTAB, 80, 5, 2, 1e-6, 1e-8, 1e-30};
    if (BiCGStabSolver<LDF>* s = dynamic_cast<BiCGStabSolver<LDF>*>(m_bottomSolver)) {
      b.imax = s->m_imax;
      b.num_restarts = s->m_numRestarts;
      b.norm_type = s->m_normType;
      b.hang = s->m_hang;
      b.small = s->m_small;
    } else if (RelaxSolver<LDF>* r = dynamic_cast<RelaxSolver<LDF>*>(m_bottomSolver)) {
      b.kind = CMG_BOTTOM_RELAX;
      b.imax = r->m_imax;
      b.num_restarts = 0;
      b.norm_type = r->m_normType;
      b.eps = r->m_eps;
      b.hang = r->m_hang;
    }
    check(cmg_set_bottom_solver(m_h, &b));
  }
  LinearSolver<LDF>* m_bottomSolver = nullptr;
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
    const cmg_solve_params p = s.params();
    GpuHierarchy::check(cmg_backward_euler(s.m_h, &p, a_dt, 1, a_zeroPhi ? 1 : 0, &st, &it));
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
    const cmg_solve_params p = s.params();
    GpuHierarchy::check(cmg_tga(s.m_h, &p, a_dt, 1, st, it));
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
