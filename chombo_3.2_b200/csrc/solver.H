// GPU AMR multigrid solver: the control flow of AMRMultiGrid::solve
// (AMRElliptic/AMRMultiGrid.H:894-1124, 1341-1419) and MultiGrid::cycle
// (AMRElliptic/MultiGrid.H:600-696) driving the device kernels, with all
// hierarchy state resident in device memory.
#ifndef CMG_SOLVER_H
#define CMG_SOLVER_H

#include <cuda_runtime.h>

#include <functional>
#include <stdexcept>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "kernels.H"
#include "plan.H"

namespace cmg {

class FineInterpOp;

struct HierarchyDesc {
  Box domain;                            // level-0 domain
  double dx0 = 1.0;                      // level-0 cell size
  std::vector<std::vector<Box>> boxes;   // per AMR level, refinement ratio 2
  int vc = 0;                            // 0: AMRPoissonOp, 1: VCAMRPoissonOp2
  double alpha = 0.0, beta = 1.0;
  int bc[6] = {0, 0, 0, 0, 0, 0};        // per domain face: 0 homogeneous Dirichlet, 1 homogeneous Neumann
  bool periodic[3] = {false, false, false};  // per direction (one-level hierarchies)
};

struct SolveParams {
  int pre = 4, post = 4, bottom = 4, numMG = 1, iterMax = 100, imin = 5;
  double eps = 1e-10, hang = 1e-10, normThresh = 1e-30;
  int iterMin = -1;  // m_iterMin: iterate at least this often whatever the norms
  // Checked on the host before the first iteration and after each one with
  // the iterations done; a non-zero return ends the solve there and is kept
  // in SolveResult::interrupted (cancellation and time limits of a server).
  std::function<int(int)> interrupt;
};

struct SolveResult {
  int exitStatus = 0, iterations = 0;
  std::vector<double> history;  // composite max-norm residual, start of each iteration, then final
  bool diverged = false;        // a residual norm was NaN or infinite (the solve stopped there)
  int interrupted = 0;          // the non-zero value SolveParams::interrupt returned, if it stopped the solve
};

// BiCGStab over the whole hierarchy preconditioned by AMR multigrid, as the
// variable-coefficient example solves (BiCGStabSolver<Vector<LevelData*>>
// over MultilevelLinearOp, VCPoissonSolve.cpp:146-183).  Defaults are the
// reference's: MultilevelLinearOp (mgIters 1, mgSmooth 4), BiCGStabSolver
// (imax 80, eps 1e-6, reps 1e-12, hang 1e-8, small 1e-30, 5 restarts) with
// the example's max norm.
struct MLSolveParams {
  int mgIters = 1, mgSmooth = 4, imax = 80, numRestarts = 5;
  double eps = 1e-6, reps = 1e-12, hang = 1e-8, small = 1e-30;
};
struct MLSolveResult {
  int exitStatus = 0, iterations = 0;  // BiCGStabSolver::m_exitStatus (1 converged, 2 rho = 0, 3 stalled), m_iter
  double initialResidual = 0, finalResidual = 0;
  std::vector<double> history;  // residual norm after each iteration
};

// Device allocation owned by the solver, stream-ordered (cudaMallocAsync /
// cudaFreeAsync on the solver's stream), so that hierarchies created and
// destroyed while others solve on their own streams never synchronise the
// device.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t s = nullptr;
  DevBuf() {}
  DevBuf(size_t n, cudaStream_t stream);
  ~DevBuf();
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

class Solver {
 public:
  Solver(const HierarchyDesc& d, cudaStream_t stream);
  // A forest of hierarchies solved together: every level and multigrid depth
  // holds the boxes of all of them (one kernel launch per operation for the
  // whole forest), each hierarchy with its own convergence test and bottom
  // solve.  Level data (setRHS, getPhi, ...) is the hierarchies' data one
  // after the other.
  Solver(const std::vector<HierarchyDesc>& descs, cudaStream_t stream);
  ~Solver();
  int numHierarchies() const { return nh_; }
  // The single-hierarchy solves and operators refuse a forest.
  void needSingle() const {
    if (nh_ > 1) throw std::invalid_argument("cmg: a forest is solved with cmg_forest_solve only");
  }
  // Valid cells of hierarchy k on level l (forest level data is ordered by
  // hierarchy).
  int64_t hierarchyCells(int k, int l) const;
  // Each hierarchy's solve, all of them advancing together: an iteration
  // runs for every hierarchy, and phi of a hierarchy whose stopping rule has
  // ended its solve is no longer changed, so each result is the one its own
  // solve gives.  Mixed: FP32 V-cycles inside FP64 refinement.
  // epsPer: a tolerance per hierarchy in place of p.eps; interrupts: a hook
  // per hierarchy (as SolveParams::interrupt, ending that hierarchy's solve).
  std::vector<SolveResult> solveForest(const SolveParams& p, bool zeroPhi, bool mixed,
                                       const std::vector<double>* epsPer = nullptr,
                                       const std::vector<std::function<int(int)>>* interrupts = nullptr);
  // fillSyntheticDevice for every hierarchy with its own seed.
  void fillSyntheticForest(const std::vector<uint64_t>& seeds);
  int numLevels() const { return (int)amr_.size(); }
  const LevelPlan& level(int l) const { return amr_[l]; }
  int numMGDepths() const { return (int)mg_.size(); }
  const LevelPlan& mgLevel(int d) const { return mg_[d]; }
  int64_t numValidCells(int l) const { return amr_[l].grids.numCells(); }
  int64_t numFaces(int l, int dir) const;
  // Valid-cell data in layout order, x fastest (host or device pointer).
  void setRHS(int l, const double* src, bool onDevice);
  void setACoef(int l, const double* src, bool onDevice);
  void setBCoef(int l, int dir, const double* src, bool onDevice);
  void getPhi(int l, double* dst, bool onDevice);
  void getRHS(int l, double* dst, bool onDevice);
  void setPhi(int l, const double* src, bool onDevice);
  // Builds lambda and the coarsened multigrid coefficients (VC operator).
  void finalizeCoefficients();
  // The seeded synthetic inputs generated on the device, coefficients
  // finalised there too (values within the last bits of the host
  // generator's, which the oracle reproduces bit for bit).
  void fillSyntheticDevice(uint64_t seed);
  SolveResult solve(const SolveParams& p, bool zeroPhi = true);
  // TGAHelmOp::setAlphaAndBeta on every operator of the hierarchy (AMR
  // levels and multigrid depths): AMRPoissonOp scales the factory's own
  // coefficients (m_alpha = alpha * aCoef, AMRPoissonOp.cpp:1103-1108),
  // VCAMRPoissonOp2 takes them as they are and recomputes lambda
  // (VCAMRPoissonOp2.cpp:258-318).
  void setAlphaAndBeta(double alpha, double beta);
  // nsteps steps of BackwardEuler::oneStep (BackwardEuler.cpp:156-189,
  // 228-245) with phi as the state and the right-hand side as the source:
  // rhs_n = a phi_n + dt src, setAlphaAndBeta(1, -dt), solve for phi_{n+1}
  // from phi_n (or from zero when zeroPhi).  The source is restored into the
  // right-hand side afterwards.  Returns each step's solve.
  std::vector<SolveResult> backwardEuler(const SolveParams& p, double dt, int nsteps, bool zeroPhi);
  // nsteps steps of AMRTGA::oneStep (AMRTGA.H:420-560), the second-order
  // Twizell-Gumel-Arigu scheme: two Helmholtz solves per step from the old
  // phi, with phi the state and the right-hand side the source (restored
  // afterwards).  Returns the 2 nsteps solves in order.
  std::vector<SolveResult> tga(const SolveParams& p, double dt, int nsteps);
  // BiCGStab over MultilevelLinearOp (see MLSolveParams) from the current
  // phi, or from zero (ghost cells included) when zeroPhi.
  MLSolveResult solveMultilevelBiCGStab(const MLSolveParams& p, bool zeroPhi = true);
  // FineInterp::interpToFine (pwc: pwcinterpToFine) of phi: every valid cell
  // of level l from phi on level l - 1 (AMRTools/FineInterp.cpp:106-160).
  void interpToFine(int l, bool pwc);
  // One composite residual evaluation (AMRMultiGrid::computeAMRResidual).
  double residualNorm();
  // The same evaluation with the max-norm reduced through `scratch`, a
  // device array of NOALLOC_MAX_BOXES + 1 doubles (noalloc.cu); allocates
  // nothing on success.
  double residualNormStatic(double* scratch);
  cudaStream_t stream() const { return s_; }
  // Runs every later call's device work on stream s (nullptr: back to the
  // hierarchy's own stream), after the work already queued has finished.
  void setStream(cudaStream_t s);
  // Device bytes held by this hierarchy.
  size_t deviceBytes() const;
  // Bytes moved per V-cycle by the algorithmic count (each array read once,
  // each output written once per pass), for the roofline.
  double vcycleBytes(const SolveParams& p) const;
  double* devPhi(int l) { return lev_[l].phi; }
  double* devRHS(int l) { return lev_[l].rhs; }

  // Per-kernel-class device timing (CUDA events around each launch of the
  // class, on the solver's stream) with the algorithmic bytes of each launch.
  // Profile classes: relaxation on the finest AMR level, residual/operator
  // kernels, ghost fills, bottom solves, relaxation on every other level.
  enum ProfClass { P_RELAX_FINE = 0, P_OP = 1, P_GHOST = 2, P_BOTTOM = 3, P_RELAX = 4, P_FINEINTERP = 5, P_NCLASS = 6 };
  void profileEnable(bool on);
  void profileRead(int cls, int64_t* launches, double* ms, double* bytes);

  template <class T>
  struct FieldsT {
    T *phi = nullptr, *rhs = nullptr, *ures = nullptr, *ucorr = nullptr, *corr = nullptr, *res = nullptr;
    T *a = nullptr, *b[3] = {nullptr, nullptr, nullptr}, *lambda = nullptr;
  };
  using LevelFields = FieldsT<double>;

  // FP32 V-cycles inside FP64 iterative refinement: the composite residual
  // with its flux-register correction, the bottom solve and the norms stay
  // FP64 (no counterpart in the reference, which is FP64 throughout).
  SolveResult solveMixed(const SolveParams& p, bool zeroPhi = true);
  // Replay each solver iteration from a CUDA graph captured on first use
  // (per precision and smoothing parameters); off by default.  Profiling
  // (profileEnable) runs the uncaptured path.
  void setUseGraphs(bool on);
  // Relaxation variant: 0 autotuned per level at the first solve (default),
  // 1 ghost fill before every colour pass, 2 face ghosts evaluated inside the
  // pass.  All three give identical results.
  void setRelaxMode(int mode);
  // Builds and uploads the fused sweep's deferred-cell lists (once).
  void ensureDeferred();
  // Builds and uploads the prefill variant's per-chunk ghost lists (once, on
  // the levels small enough for them).
  void ensureChunkGhosts();
  // The bottom solver of the multigrid levels below level 0 (BottomConfig).
  // Host seconds of the constructor: plan building, then device set-up
  // (allocation, uploads, coefficient fills); 0 for a forest.
  double planSeconds() const { return planSeconds_; }
  double deviceSeconds() const { return deviceSeconds_; }
  void setBottomConfig(const BottomConfig& c);
  // How the bottom solve runs: -1 automatic (the whole device for one
  // hierarchy whose bottom level has at least kBottomGridMinCells cells,
  // else one block per hierarchy), 0 one block, 1 the whole device (one
  // hierarchy only).  The results are the same bit for bit.
  void setBottomGrid(int mode);
  bool bottomOnGrid() const { return bottomGrid_ > 0; }
  static constexpr int kBottomGridMinCells = 4096;
  const BottomConfig& bottomConfig() const { return bottomCfg_; }
  // The variant of every AMR level then every multigrid depth (1: inline),
  // and the tuner's sweep times (ms; empty when a mode was forced).
  void relaxVariants(std::vector<int>& inl, std::vector<float>& msFill, std::vector<float>& msInline);

  // Operator-level calls (levelops.cu): one AMRLevelOp / MGLevelOp / LinearOp
  // method of one level on host arrays in the ghosted box format (every
  // box's FAB grown by one cell, x fastest, boxes in layout order).  lev >= 0
  // is an AMR level, lev < 0 the multigrid depth -lev below level 0.  Inputs
  // are read whole; outputs get their valid cells written (ghost positions
  // unspecified).  Each call synchronises the solver's stream.
  const LevelPlan& opPlan(int lev) const;
  int64_t opSize(int lev) const;          // doubles in one ghosted array of lev
  int64_t opCoarsenedSize(int l) const;   // doubles in one ghosted array of coarsen(level l, 2)
  void opResidual(int lev, double* lhs, const double* phi, const double* rhs, bool homogeneous);
  void opApply(int lev, double* lhs, const double* phi, bool homogeneous);
  void opRelax(int lev, double* phi, const double* rhs, int iterations);
  void opPreCond(int lev, double* cor, const double* res);
  void opRestrictResidual(int lev, double* resCoarse, const double* phi, const double* rhs);
  void opProlongIncrement(int lev, double* phi, const double* corrCoarse);
  void opAMROperator(int l, double* out, const double* phiFine, double* phi, const double* phiCoarse,
                     const double* rhs, int form);
  void opAMRRestrict(int l, double* resCoarsened, const double* residual, const double* corr,
                     const double* corrCoarse);
  void opAssignCoarsened(int l, double* coarse, const double* coarsened);
  void opAMRProlong(int l, double* corr, const double* corrCoarse);
  void opAMRUpdateResidual(int l, double* res, const double* corr, const double* corrCoarse);
  void opZeroCovered(int l, double* data);
  void opCFInterp(int l, double* phi, const double* phiCoarse);
  void opAxby(int lev, double* lhs, const double* x, const double* y, double a, double b);
  void opIncr(int lev, double* lhs, const double* x, double scale);
  void opScale(int lev, double* lhs, double scale);
  double opDot(int lev, const double* x, const double* y);
  double opNorm(int lev, const double* x, int p);

 private:
  // Device state of the operator-level calls of one level.
  struct OpState {
    static constexpr int kFields = 5;
    int64_t size = 0, csize = 0;                // ghosted and coarsened-fine ghosted doubles
    const int64_t* off = nullptr;               // per box: first element in the ghosted format
    const int64_t* coff = nullptr;              // the same in the coarsened-fine format
    double *packed = nullptr, *packed2 = nullptr, *packed3 = nullptr;  // host-format staging
    double* field[kFields] = {};                // level-sized device fields
  };
  std::map<int, std::unique_ptr<OpState>> opStates_;
  OpState& opState(int lev);
  double* opField(int lev, int k);
  void* uploadRaw(const void* src, size_t bytes);
  double* opLoad(int lev, int k, const double* host);
  void opStore(int lev, const double* f, double* host);
  void opStoreGrown(int lev, const double* f, double* host);
  void opEnsureTuned();
  std::vector<double> opBoxValues(int lev, int nbox);
  const LevelDev& opDev(int lev) const;
  Coef<double> opCoef(int lev) const;

  void uploadLevel(const LevelPlan& p, LevelDev& d);
  double* alloc(size_t n);
  Coef<double> coefAMR(int l) const;
  Coef<double> coefMG(int d) const;
  // The V-cycle in precision T (double: the drop-in; float: the inner
  // cycles of solveMixed).
  template <class T> std::vector<FieldsT<T>>& levF();
  template <class T> std::vector<FieldsT<T>>& mgF();
  template <class T> Coef<T> coefA(int l);
  template <class T> Coef<T> coefM(int d);
  template <class T> void relaxAMR(int l, T* phi, const T* rhs, int n);
  template <class T> void relaxMG(int d, T* phi, const T* rhs, int n);
  template <class T>
  void relaxLevel(const LevelDev& L, double cells, const Coef<T>& c, T* phi, const T* rhs, int n, int cls,
                  int variant);
  // Levels up to this many cells may relax all sweeps in one one-block launch.
  static constexpr double kBlockRelaxMaxCells = 32768;
  // Relaxation variants: 0 ghost fill before each colour pass, 1 face ghosts
  // in the pass, 2 every sweep in one one-block launch, 3 fused sweeps
  // (gsrbSweepFused: both colours per launch, boxes marching in z).
  static constexpr int kRelaxVariants = 4;
  template <class T> void fill(const LevelDev& L, T* f, bool withCF, int par = -1);
  template <class T>
  void amrResidualLevel(int ilev, int lmax, T* const* res, T* const* phi, T* const* rhs);
  double computeAMRResidual(std::vector<double*>& res, std::vector<double*>& phi, std::vector<double*>& rhs, int lmax);
  void launchAMRResidual(std::vector<double*>& res, std::vector<double*>& phi, std::vector<double*>& rhs, int lmax);
  double readNorm();
  std::vector<double> readNorms();  // one per hierarchy
  SolveResult solveImpl(const SolveParams& p, bool zeroPhi, bool mixed);
  void iterationBody(bool mixed, std::vector<double*>& ures, std::vector<double*>& phi, std::vector<double*>& rhs);
  cudaGraphExec_t iterationGraph(bool mixed, std::vector<double*>& ures, std::vector<double*>& phi,
                                 std::vector<double*>& rhs);
  // Captured graphs hold the operator coefficients as kernel arguments, so
  // alpha and beta are part of the key (setAlphaAndBeta switches between
  // captured graphs instead of recapturing).
  struct GraphKey {
    bool mixed;
    int pre, post, bottom, numMG;
    double eps, alpha, beta;
    bool operator<(const GraphKey& o) const {
      if (mixed != o.mixed) return mixed < o.mixed;
      if (pre != o.pre) return pre < o.pre;
      if (post != o.post) return post < o.post;
      if (bottom != o.bottom) return bottom < o.bottom;
      if (numMG != o.numMG) return numMG < o.numMG;
      if (eps != o.eps) return eps < o.eps;
      if (alpha != o.alpha) return alpha < o.alpha;
      return beta < o.beta;
    }
  };
  static constexpr size_t kMaxGraphs = 16;  // cache bound (a new key past it drops the cache)
  std::map<GraphKey, cudaGraphExec_t> graphs_;
  std::map<cudaGraphExec_t, long long> graphLaunches_;  // kernel launches per replay
  bool useGraphs_ = false;
  // Relaxation variant per AMR level / MG depth: ghost fill before each
  // colour pass (0), face ghosts evaluated inside the pass (1), every sweep
  // in one one-block launch with in-pass ghosts (2), or fused sweeps (3).
  std::vector<char> inlineA_, inlineM_;
  bool tuned_ = false;
  int relaxMode_ = 0;  // 0: autotuned, 1: always fills, 2: always inline, 3: always fused
  std::vector<std::pair<float, float>> tuneMs_;
  void tuneRelaxation();
  double* hostScalars_ = nullptr;  // pinned: [0] norm read back, [1] bottom metric
  template <class T> void amrVCycle(int ilev, int lmax);
  template <class T> void mgCycle(int depth, T* corr, T* res);
  template <class T> void bottom(int depth, T* corr, T* res);
  template <class T> void zeroField(const LevelDev& L, T* f);
  template <class T> void copyField(const LevelDev& L, T* dst, const T* src);
  void ensure32();
  float* allocF(size_t n);
  // MultilevelLinearOp on device vectors (one array per AMR level).
  using MLVec = std::vector<double*>;
  double alpha0_ = 0.0, beta0_ = 1.0;  // the factory's coefficients (AMRPoissonOp m_aCoef, m_bCoef)
  std::vector<double*> src_;           // backward-Euler source per level
  std::vector<std::unique_ptr<FineInterpOp>> fineInterp_;  // per fine level, built on first use
  std::vector<MLVec> mlVecs_;    // r, r_tilde, e, p, p_tilde, s_tilde, t, v, and two scratch vectors
  double* dBoxSums_ = nullptr;   // one per box of every level
  double* hostBoxSums_ = nullptr;
  MLVec mlVec(int i);
  void mlZero(MLVec& x);
  void mlAssign(MLVec& dst, const MLVec& src);
  void mlIncr(MLVec& y, const MLVec& x, double scale);
  void mlScale(MLVec& x, double scale);
  void mlResidual(MLVec& lhs, MLVec& phi, MLVec& rhs);
  void mlApplyOp(MLVec& lhs, MLVec& phi);
  double mlNorm(const MLVec& x);
  double mlDot(const MLVec& x, const MLVec& y);
  void mlPreCond(MLVec& cor, MLVec& res, const MLSolveParams& p);
  void mlPreCondBody(MLVec& cor, MLVec& res, const MLSolveParams& p);
  // Captured preconditioner calls, per (correction, residual) vector pair and
  // smoothing parameters.
  std::map<std::tuple<const void*, const void*, int, int, double, double>, cudaGraphExec_t> precondGraphs_;
  void amrOperatorLevel(int ilev, int lmax, MLVec& lhs, MLVec& phi);
  void scatterValid(const LevelPlan& p, const LevelDev& d, double* dev, const double* src, bool onDevice,
                    int faceDir);
  void gatherValid(const LevelPlan& p, const LevelDev& d, const double* dev, double* dst, bool onDevice);
  struct RegionPlan {
    int n = 0;
    int64_t total = 0;
    const void* dev = nullptr;
  };
  std::map<std::pair<const void*, int>, RegionPlan> regionCache_;
  const void* regionPlan(const LevelPlan& p, int faceDir, int* nreg, int64_t* total);
  std::unique_ptr<DevBuf> stage_;
  double* staging(int64_t n);

  cudaStream_t s_;    // stream of the device work
  cudaStream_t own_;  // the hierarchy's own stream: every allocation and free
  void ownSync();     // completes pending allocations before s_ uses them
  HierarchyDesc desc_;
  std::vector<LevelPlan> amr_;
  std::vector<LevelPlan> mg_;        // multigrid depths below level 0; mg_[0] is depth 1
  std::vector<LevelDev> amrDev_, mgDev_;
  std::vector<LevelFields> lev_;
  std::vector<LevelFields> mgf_;     // corr, res and coefficients per depth
  std::vector<FieldsT<float>> lev32_, mgf32_;  // FP32 V-cycle fields (allocated on first solveMixed)
  bool have32_ = false, coef32Stale_ = true;
  std::vector<std::unique_ptr<DevBuf>> bufs_;
  std::vector<BottomWork> bottoms_;         // one per hierarchy (one unless a forest)
  const BottomWork* dBottoms_ = nullptr;    // the same in device memory
  int maxBottomBoxes_ = 1;
  int bottomGrid_ = 0;
  double planSeconds_ = 0, deviceSeconds_ = 0;  // blocks of the grid-wide bottom solve, 0 for one block per hierarchy
  BottomConfig bottomCfg_;
  int nh_ = 1;                              // hierarchies (a forest: more than one)
  int* dActive_ = nullptr;                  // per hierarchy: still iterating (forest solves)
  double* dEps_ = nullptr;                  // per hierarchy: bottom-solver tolerance (forest solves)
  int* hostActive_ = nullptr;               // pinned staging of dActive_
  void setup(const std::vector<BottomPlan>& bps);
  double* dNorm_ = nullptr;
  int64_t bottomCells_ = 0;
  SolveParams sp_;
  double* dMetric_ = nullptr;  // bottom solver's convergence metric (device)
  std::vector<std::vector<double>> hostA_, hostB_[3];

  struct ProfRec {
    cudaEvent_t a, b;
    int cls;
    double bytes;
  };
  bool profOn_ = false;
  std::vector<ProfRec> prof_;
  std::vector<cudaEvent_t> evPool_;
  cudaEvent_t takeEvent();
  template <class F>
  void timed(int cls, double bytes, F f) {
    if (!profOn_) return f();
    ProfRec r{takeEvent(), takeEvent(), cls, bytes};
    cudaEventRecord(r.a, s_);
    f();
    cudaEventRecord(r.b, s_);
    prof_.push_back(r);
  }
  double profAcc_[P_NCLASS][3] = {};
  void profileDrain();
};

}  // namespace cmg

#endif
