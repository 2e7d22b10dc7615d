// Device kernels of the AMR multigrid V-cycle (sm_100a).  Each launcher
// applies one reference operation to every box of a level in one launch,
// driven by the tables in devtypes.H.  T is the field precision (double for
// the drop-in solve, float for the inner V-cycles of iterative refinement).
#ifndef CMG_KERNELS_H
#define CMG_KERNELS_H

#include <cuda_runtime.h>

#include "devtypes.H"

namespace cmg {

// Device-resident plan of one level (pointers into device memory).
struct LevelDev {
  const BoxDesc* boxes = nullptr;
  int nbox = 0;
  int64_t nelem = 0;
  const GhostTaskDev* ghost = nullptr;
  int nExchBC = 0, nGhost = 0;
  const int* ghostStart = nullptr;       // cumulative cell counts (nGhost + 1)
  const int* ghostBlock = nullptr;       // first task of each GHOST_PER_BLOCK cells
  const int* slotStart = nullptr;        // the same over one-colour slots
  const int* slotBlock = nullptr;
  int nSlotsExchBC = 0, nSlotsGhost = 0;
  int nCellsExchBC = 0, nCellsGhost = 0;
  const GhostCell* gcells = nullptr;     // flat ghost-cell lists (LevelPlan::gcells)
  int gcStart[2] = {0, 0}, gcExch[2] = {0, 0}, gcCF[2] = {0, 0};
  // forest levels (several hierarchies, LevelPlan::boxHier / hierStart):
  // hierarchy of each box and first element of each hierarchy; null and 1
  // for one hierarchy
  const int* boxHier = nullptr;
  const int64_t* hierStart = nullptr;
  int nh = 1;
  const FaceRule* faceRules = nullptr;    // LevelPlan::faceRules / faceOff
  const int* faceOff = nullptr;
  const DeferredCell* deferred = nullptr; // LevelPlan::deferred
  int nDeferred = 0;
  const GhostCell* chGhost[2] = {nullptr, nullptr};  // LevelPlan::chunkGhost
  const int* chGhostStart[2] = {nullptr, nullptr};
  const GhostTaskDev* zero = nullptr;
  int nZero = 0;
  const int* zeroStart = nullptr;
  const int* zeroBlock = nullptr;
  int nCellsZero = 0;
  const Chunk* chAll = nullptr;
  int nAll = 0;
  const Chunk* chColor[2] = {nullptr, nullptr};
  int nColor[2] = {0, 0};
  // coarse-fine interpolation from the coarser level
  const CFCoarse* cfC = nullptr;
  const CFFine* cfF = nullptr;
  int nCfF = 0;
  int nCfC = 0;                 // coarse cells of the interpolation (cfC entries)
  double* cfTmp = nullptr;      // 6 values per cfC entry (derivatives and the coarse value), T-typed
  const double* cfW = nullptr;
  const int64_t* cfOff = nullptr;
  // coarse/fine maps to the coarser level
  const CoarseFineItem* items = nullptr;
  const Chunk* itemChC = nullptr;
  int nItemChC = 0;
  const Chunk* itemChF = nullptr;
  int nItemChF = 0;
  // flux-register correction from the finer level
  const RefluxCell* rfCells = nullptr;
  int nRf = 0;
  const RefluxCoarseTerm* rfC = nullptr;
  const RefluxFineGroup* rfF = nullptr;
  double dx = 0, dxCrse = 0;
};

// Operator coefficients: L = alpha*phi + beta*Lap(phi) (constant, vc = 0) or
// L = alpha*a*phi - beta*div(b grad phi) (variable, vc = 1).
template <class T>
struct Coef {
  int vc = 0;
  double alpha = 0, beta = 1;
  const T* a = nullptr;
  const T* b[3] = {nullptr, nullptr, nullptr};
  const T* lambda = nullptr;
};

// Ghost fill: exchange copies and physical BC values, plus the homogeneous
// coarse-fine values when withCF; par >= 0 restricts it to ghost cells of
// colour par (the only ones a pass over colour 1 - par reads).
template <class T> void ghostFill(const LevelDev& L, T* f, bool withCF, cudaStream_t s, int par = -1);
template <class T> void zeroCovered(const LevelDev& L, T* f, cudaStream_t s);
// Backward-Euler right-hand side over a whole level array:
// rhs = ((0 + phi) * a) + ((0 + src) * dt), a == nullptr for no a-coefficient.
void eulerRHS(double* rhs, const double* phi, const double* a, const double* src, double dt, int64_t n,
              cudaStream_t s);
// TGA source term over a whole level array: out = (0 + src * 1) / a (no
// division when a == nullptr).
void tgaSource(double* out, const double* src, const double* a, int64_t n, cudaStream_t s);
// x *= a elementwise over a whole level array.
void multField(double* x, const double* a, int64_t n, cudaStream_t s);
// x *= scale over a whole level array.
void scaleField(double* x, double scale, int64_t n, cudaStream_t s);
// out[b] = sum of x*y over the valid cells of box b, accumulated in the
// reference's order (FArrayBox::dotProduct: k, j, i with i fastest).
void boxDots(const LevelDev& L, const double* x, const double* y, double* out, cudaStream_t s);
// One colour pass of levelGSRB.  inlineGhosts: every block first writes the
// face ghosts its own cells read (LevelDev::chGhost, the entries of the fill
// that would precede the pass), so no ghost fill is needed before the pass;
// otherwise they are read from ghost cells filled by ghostFill(withCF) just
// before.
template <class T>
void gsrb(const LevelDev& L, T* phi, const T* rhs, const Coef<T>& c, int color, cudaStream_t s,
          bool inlineGhosts = false);
// One whole red-black sweep (both colours) in two launches: every box
// marches through its z slabs updating the colour-0 cells of slab k and then
// the colour-1 cells of slab k - 1, each face coefficient and neighbour read
// once for both colours; the face ghosts come from the level's fill rules
// (no fill).  The colour-1 cells on exchange faces need other boxes' new
// colour-0 values and are updated by the second launch (LevelDev::deferred).
// Same values as gsrb() for colour 0 then colour 1.
template <class T>
void gsrbSweepFused(const LevelDev& L, T* phi, const T* rhs, const Coef<T>& c, cudaStream_t s);
// nsweeps red-black sweeps of a small level in a single one-block launch
// (in-pass ghosts, block barriers between colour passes); same results.
template <class T>
void relaxBlock(const LevelDev& L, T* phi, const T* rhs, const Coef<T>& c, int nsweeps, cudaStream_t s);
// residualI form: r = rhs - L(phi) in the operator's own expression order.
template <class T> void residual(const LevelDev& L, T* r, const T* phi, const T* rhs, const Coef<T>& c, cudaStream_t s);
// applyOpI form: lofphi = L(phi).
template <class T> void applyOp(const LevelDev& L, T* lofphi, const T* phi, const Coef<T>& c, cudaStream_t s);
// r = -lofphi + rhs (LevelDataOps::axby(r, r, rhs, -1, 1)); valid cells as the
// reference, ghost slots overwritten too (they are refilled before any read).
template <class T> void negAdd(const LevelDev& L, T* r, const T* lofphi, const T* rhs, cudaStream_t s);
// Multigrid restriction of the residual (RESTRICTRES), box b -> coarsened box b.
template <class T> void restrictMG(const LevelDev& F, const LevelDev& C, T* resC, const T* phi, const T* rhs,
                                   const Coef<T>& c, cudaStream_t s);
// Multigrid piecewise-constant prolongation, box b <- coarsened box b.
template <class T> void prolongMG(const LevelDev& F, const LevelDev& C, T* phi, const T* corrC, cudaStream_t s);
// AMR restriction: coarse(c) = average of 8 fine values, over coarse/fine items.
template <class T> void averageAMR(const LevelDev& F, const LevelDev& C, T* coarse, const T* fine, cudaStream_t s);
// AMR prolongation: fine += coarse(i/2) over coarse/fine items.
template <class T> void prolongAMR(const LevelDev& F, const LevelDev& C, T* fine, const T* coarse, cudaStream_t s);
// Inhomogeneous quadratic coarse-fine ghost fill of phiF from phiC.
template <class T> void quadCF(const LevelDev& F, T* phiF, const T* phiC, cudaStream_t s);
// Flux-register correction of lofphiC from phiC and phiF (finer level).
template <class T> void reflux(const LevelDev& C, T* lofphiC, const T* phiC, const T* phiF, const Coef<T>& cc,
                               const Coef<T>& cf, cudaStream_t s);
// lhs += scale * x (LevelDataOps::incr); valid cells as the reference, ghost
// slots too (refilled before any read).
template <class T> void incr(const LevelDev& L, T* lhs, const T* x, double scale, cudaStream_t s);
// lhs += x, then x = lhs (the increment and the copy back of AMRVCycle's
// post-smoothing), in one pass over whole level arrays.
template <class T> void incrCopy(const LevelDev& L, T* lhs, T* x, cudaStream_t s);
// lhs += x, then x = 0, in one pass over whole level arrays.
template <class T> void incrZero(const LevelDev& L, T* lhs, T* x, cudaStream_t s);
// lhs += x over valid cells, an FP32 correction added to an FP64 field.
void incrMixed(const LevelDev& L, double* lhs, const float* x, cudaStream_t s);
// dst[q] = src[q] for every element of a level array (valid and ghost cells).
template <class D, class S> void convert(D* dst, const S* src, int64_t n, cudaStream_t s);
// Max |f| over valid cells, folded into *out (device scalar) with max();
// on a forest level into out[k] for each hierarchy k.
template <class T> void maxNorm(const LevelDev& L, const T* f, double* out, cudaStream_t s);
// lhs += x (flat, like incr / incrMixed) on the element ranges of the
// hierarchies k of a forest level with active[k] != 0 only.
template <class T, class X>
void incrActive(const LevelDev& L, T* lhs, const X* x, const int* active, cudaStream_t s);

// Bottom BiCGStab state in the compact slot space of the bottom level
// (BottomPlan): slot tables, vectors r, r~, e, p, p~, s~, t, v, phi, rhs
// (nv + ng doubles each), the compact coefficients of a variable-coefficient
// operator, and a 2-int status (exit, iterations).
// Which bottom solver runs and its public parameters: BiCGStabSolver
// (BiCGStabSolver.H:165-182 defaults; its eps comes from the multigrid
// solver's convergence metrics) or RelaxSolver (RelaxSolver.H:104-112
// defaults, its own eps).  normType 2 or 0.
struct BottomConfig {
  int kind = 0;  // 0 BiCGStabSolver, 1 RelaxSolver
  int imax = 80, numRestarts = 5, normType = 2;
  double eps = 1e-6, hang = 1e-8, small = 1e-30, reps = 1e-12;
};
struct BottomWork {
  int nv = 0, ng = 0, nbox = 0, ncol[2] = {0, 0};
  int maxBoxCells = 0;  // cells of the largest box
  const int *fab = nullptr, *nb = nullptr, *col[2] = {nullptr, nullptr}, *boxStart = nullptr;
  const int* nbv = nullptr;  // 6 per valid slot: face neighbour value source (BottomPlan::nbv)
  double* v[10] = {};
  double *a = nullptr, *b[3] = {nullptr, nullptr, nullptr}, *lam = nullptr;
  int* status = nullptr;
  double *gpart = nullptr, *gpart2 = nullptr, *gscal = nullptr;  // sums of a grid-wide solve
};
// Bottom solve (BiCGStab or relaxation, cfg) of L(phi) = rhs (homogeneous
// boundary conditions) on one level, one thread block per hierarchy
// (works[0 .. nworks), device memory; several for a forest), reference
// summation order.  eps and metrics[k] are the tolerance and convergence
// metric AMRMultiGrid hands hierarchy k's bottom solver (the metric read
// from device memory when the kernel runs, so a captured launch serves every
// solve).  phi and rhs are level fields; the coefficients come from the
// works.  maxBoxes: the largest box count of a work.  epsPer (device, may be
// null): a BiCGStab tolerance per hierarchy in place of eps.  gridBlocks > 0
// (one work only, its gpart/gpart2/gscal set): the whole solve as one
// cooperative launch of that many blocks instead of one block.
void bottomSolve(const LevelDev& L, double* phi, const double* rhs, const Coef<double>& c, const BottomWork* works,
                 int nworks, int maxBoxes, const BottomConfig& cfg, double eps, const double* metrics,
                 cudaStream_t s, const double* epsPer = nullptr, int gridBlocks = 0);
// Blocks of a grid-wide bottom solve of nv valid cells (bounded by what is
// co-resident on the device), and threads per block.
int bottomGridBlocks(int nv);
int bottomGridThreads();
// dst[slot] = fab[w.fab[slot]] for every slot of the bottom level.
void gatherSlots(const BottomWork& w, const double* fab, double* dst, cudaStream_t s);

// Seeded synthetic inputs of one level on the device (rhs; a and the three
// face arrays b when not null), the same formulas as synthetic.H.
void fillSyntheticLevel(const LevelDev& L, uint64_t seed, double* rhs, double* a, double* const b[3],
                        cudaStream_t s);
// The same over boxes [box0, box1) whose chunks are [ch0, ch1) of L.chAll
// (one hierarchy of a forest level).
void fillSyntheticBoxes(const LevelDev& L, uint64_t seed, double* rhs, double* a, double* const b[3], int box0,
                        int box1, int ch0, int ch1, cudaStream_t s);
// lambda of the variable-coefficient relaxation on one level
// (VCAMRPoissonOp2::resetLambda with SUMFACES).
void lambdaLevel(const LevelDev& L, const double* a, const double* const b[3], double alpha, double beta,
                 double* lam, cudaStream_t s);
// a and b of multigrid level C averaged from level F by ratio r, box b <- box b
// (CoarseAverage / CoarseAverageFace arithmetic).
void averageCoefficients(const LevelDev& F, const LevelDev& C, int r, const double* fa, const double* const fb[3],
                         double* ca, double* const cb[3], cudaStream_t s);

// Number of kernel launches issued by the launchers above since load.
long long launchCount();
// Counts n launches that ran without passing through the launchers (the
// kernel nodes of a replayed CUDA graph).
void addLaunches(long long n);

}  // namespace cmg

#endif
