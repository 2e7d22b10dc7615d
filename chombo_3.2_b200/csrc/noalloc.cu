// Composite residual max-norm that allocates nothing.
//
// cmg_residual_norm reduces into a device scalar the hierarchy allocated
// and gathers its level pointers in host vectors.  Some callers cannot let a
// library allocate at call time: a serving process that has handed all free
// HBM to its own memory pool (a cudaMalloc on the side can then fail, or make
// the pool release cached blocks and synchronise the device), and a
// latency-bound monitoring loop that checks the residual between solves
// (cudaMalloc and cudaFree synchronise the device).  This variant keeps its
// reduction scratch in a fixed array of this file, g_normScratch, and uses no
// heap memory on its success path: the residual itself goes to the
// hierarchy's own residual arrays, allocated once when the hierarchy was
// built, exactly as cmg_residual_norm does.
//
// Limits and rules of use:
//  - the scratch holds one partial maximum per box of a level, so a level
//    may have at most NOALLOC_MAX_BOXES boxes (larger calls are rejected),
//    and the hierarchy at most NOALLOC_MAX_LEVELS levels;
//  - the first call on a device looks the scratch up with
//    cudaGetSymbolAddress while that device is current; make that first call
//    before any stream capture begins on the device;
//  - the running-maximum slot must start at zero: every call zeroes it on
//    its stream before the first level; the per-box slots need no initial
//    value (each slot is written before it is read in the same call);
//  - all calls on one device share the scratch: calls that overlap in time
//    (two host threads, or two hierarchies on unordered streams) race on it
//    and may return each other's values, so serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "noalloc.H"
#include "solver.H"

namespace cmg {

static_assert(NOALLOC_MAX_BOXES == 4096 && NOALLOC_MAX_LEVELS == 16, "limits quoted in the messages below");

namespace {

// [0, NOALLOC_MAX_BOXES): per-box maxima of the level being reduced;
// [NOALLOC_MAX_BOXES]: running maximum over the levels done so far.
__device__ __align__(256) double g_normScratch[NOALLOC_MAX_BOXES + 1];

std::mutex g_setupMutex;
double* g_scratchPtr[NOALLOC_MAX_DEVICES] = {};

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    // Error path only: the message string is built after the failure.
    throw std::runtime_error(std::string("cmg: ") + what + ": " + cudaGetErrorString(e));
  }
}

// Device address of the scratch for device `dev`, which must be current.
double* scratchFor(int dev) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    throw std::invalid_argument("cmg: residual_norm_noalloc: device ordinal beyond the scratch table");
  std::lock_guard<std::mutex> lock(g_setupMutex);
  if (!g_scratchPtr[dev]) {
    double* ptr = nullptr;
    ck(cudaGetSymbolAddress((void**)&ptr, g_normScratch), "cudaGetSymbolAddress");
    g_scratchPtr[dev] = ptr;
  }
  return g_scratchPtr[dev];
}

}  // namespace

void forgetNoAllocScratch() {
  std::lock_guard<std::mutex> lock(g_setupMutex);
  for (double*& p : g_scratchPtr) p = nullptr;
}

namespace {

enum { NT = 256 };

// max(a, b) that keeps a NaN from either side (fmax drops it), so that a
// residual holding a NaN reduces to NaN.
__device__ __forceinline__ double nanMax(double a, double b) { return (b > a || b != b) ? b : a; }

__device__ __forceinline__ double blockMax(double v) {
  __shared__ double red[NT / 32];
  for (int o = 16; o > 0; o >>= 1) v = nanMax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = nanMax(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

// One block per box: max |f| over the box's valid cells into part[box].
// Same value as the atomic k_maxnorm (a maximum does not depend on order).
__global__ void __launch_bounds__(NT) k_boxmax(const BoxDesc* boxes, const double* f, double* part) {
  const BoxDesc bd = boxes[blockIdx.x];
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1, nz = bd.hi[2] - bd.lo[2] + 1;
  const int n = nx * ny * nz;
  double v = 0.0;
  for (int q = threadIdx.x; q < n; q += NT) {
    int i = bd.lo[0] + q % nx, r = q / nx, j = bd.lo[1] + r % ny, k = bd.lo[2] + r / ny;
    v = nanMax(v, fabs(f[cellIndex(bd, i, j, k)]));
  }
  v = blockMax(v);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// One block: fold the per-box maxima of a level into the running maximum.
__global__ void __launch_bounds__(NT) k_foldmax(const double* part, int nbox, double* acc) {
  double v = 0.0;
  for (int b = threadIdx.x; b < nbox; b += NT) v = nanMax(v, part[b]);
  v = blockMax(v);
  if (threadIdx.x == 0) *acc = nanMax(*acc, v);
}

// Makes the stream's device current for the lifetime of the object.
struct DeviceScope {
  int prev = -1, dev = -1;
  explicit DeviceScope(cudaStream_t s) {
    ck(cudaStreamGetDevice(s, &dev), "cudaStreamGetDevice");
    ck(cudaGetDevice(&prev), "cudaGetDevice");
    if (prev != dev) ck(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DeviceScope() {
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  }
};

}  // namespace

// AMRMultiGrid::computeAMRResidual (AMRMultiGrid.H:682-736) with the same
// kernels and order as Solver::computeAMRResidual, level pointers kept on
// the stack and the max-norm reduced through the static scratch.
double Solver::residualNormStatic(double* scratch) {
  needSingle();
  const int nlev = numLevels(), lmax = nlev - 1;
  if (nlev > NOALLOC_MAX_LEVELS)
    throw std::invalid_argument("cmg: residual_norm_noalloc: more than 16 levels (static scratch limit)");
  for (int l = 0; l < nlev; ++l)
    if (amrDev_[l].nbox > NOALLOC_MAX_BOXES)
      throw std::invalid_argument(
          "cmg: residual_norm_noalloc: a level has more than 4096 boxes (static scratch limit)");
  double* res[NOALLOC_MAX_LEVELS];
  double* phi[NOALLOC_MAX_LEVELS];
  double* rhs[NOALLOC_MAX_LEVELS];
  for (int l = 0; l < nlev; ++l) {
    res[l] = lev_[l].res;
    phi[l] = lev_[l].phi;
    rhs[l] = lev_[l].rhs;
  }
  double* acc = scratch + NOALLOC_MAX_BOXES;
  ck(cudaMemsetAsync(acc, 0, sizeof(double), s_), "scratch reset");
  for (int ilev = 0; ilev <= lmax; ++ilev) {
    const LevelDev& L = amrDev_[ilev];
    // The composite residual of the level, by the same code as every solve.
    amrResidualLevel<double>(ilev, lmax, res, phi, rhs);
    if (ilev != lmax) zeroCovered(L, res[ilev], s_);
    if (L.nbox == 0) continue;
    k_boxmax<<<L.nbox, NT, 0, s_>>>(L.boxes, res[ilev], scratch);
    ck(cudaGetLastError(), "k_boxmax");
    k_foldmax<<<1, NT, 0, s_>>>(scratch, L.nbox, acc);
    ck(cudaGetLastError(), "k_foldmax");
  }
  double h = 0;
  ck(cudaMemcpyAsync(&h, acc, sizeof(double), cudaMemcpyDeviceToHost, s_), "norm d2h");
  ck(cudaStreamSynchronize(s_), "norm sync");
  return h;
}

double residualNormNoAlloc(Solver& S) {
  DeviceScope scope(S.stream());
  return S.residualNormStatic(scratchFor(scope.dev));
}

}  // namespace cmg
