// FineInterp on the device (fineinterp.H).  Bit-exact with the reference:
// compiled with --fmad=false, every slope, limiter and fine value is formed
// with the reference's operations in its order (InterpF.ChF:48-71, 135-312,
// 318-369).
//
// Two paths.  When every fine box's staging block (its coarsened box grown by
// one) fits in shared memory, one kernel does everything: a thread block per
// fine box loads the block from the coarse level, then computes and stores
// the box's fine cells.  Otherwise a gather kernel fills per-box staging
// blocks in device memory and a second kernel interpolates from them.
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "fineinterp.H"
#include "kernels.H"

namespace cmg {

namespace {

constexpr int kChunk = 256;
constexpr int kFusedThreads = 256;
constexpr int kLoadILP = 8;
constexpr int kSeg = 8;  // planes per work item of the one-kernel path
constexpr size_t kFusedSmemMax = 96 * 1024;  // staging bytes per block on the one-kernel path

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "cmg: %s: %s", what, cudaGetErrorString(e));
    throw std::runtime_error(buf);
  }
}

void chunks(std::vector<Chunk>& out, int item, int64_t n) {
  for (int64_t s = 0; s < n; s += kChunk) out.push_back(Chunk{item, (int)s});
}

// The fine cells of one box addressed from a base: cell (2i + c0, 2j + c1,
// 2k + c2), (i, j, k) local to the coarsened box, is at(lin(i, j, k) + c0 +
// dy c1 + dz c2, (c0 + c1 + c2) & 1).
struct FineRB {  // red-black level field (colourSlot / cellIndex)
  int64_t off, half;
  int dy, dz;
  __device__ __forceinline__ int lin(int i, int j, int k) const { return (2 * i + 1) + dy * (2 * j + 1) + dz * (2 * k + 1); }
  __device__ __forceinline__ int64_t at(int l, int colour) const { return off + colour * half + (l >> 1); }
};
struct FineFlat {  // flat valid-cell array
  int64_t off;
  int dy, dz;
  __device__ __forceinline__ int lin(int i, int j, int k) const { return 2 * i + dy * 2 * j + dz * 2 * k; }
  __device__ __forceinline__ int64_t at(int l, int) const { return off + l; }
};

// Element index of cell (i, j, k) of box `box` in a red-black level field.
struct RBCells {
  const BoxDesc* b;
  __device__ __forceinline__ int64_t operator()(int box, int i, int j, int k) const {
    return cellIndex(b[box], i, j, k);
  }
  __device__ __forceinline__ FineRB rows(int box) const {
    const BoxDesc x = b[box];
    return FineRB{x.off, x.half, x.px, x.px * x.py};
  }
};

// ... in a flat valid-cell array.
struct FlatCells {
  const FlatBox* b;
  __device__ __forceinline__ int64_t operator()(int box, int i, int j, int k) const {
    const FlatBox& x = b[box];
    return x.off + (i - x.lo[0]) + (int64_t)x.nx * ((j - x.lo[1]) + (int64_t)x.ny * (k - x.lo[2]));
  }
  __device__ __forceinline__ FineFlat rows(int box) const {
    const FlatBox x = b[box];
    return FineFlat{x.off, x.nx, x.nx * x.ny};
  }
};

// Extrema of the 3 x 3 cells around p in its plane (row stride sy).
__device__ __forceinline__ void planeExtrema(const double* p, int sy, double& mx, double& mn) {
  mx = p[0];
  mn = p[0];
#pragma unroll
  for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
    for (int di = -1; di <= 1; ++di) {
      const double w = p[di + dj * sy];
      mx = fmax(mx, w);
      mn = fmin(mn, w);
    }
}

// Coarse cell (I, J, K) of b, its staging value at s (strides sy, sz): the
// eight fine cells.  interpconstant, then on b_mod the central slopes
// (interpcentralslope), the limiter (interplimit) and the three linear
// corrections (interplinear, dir 0, 1, 2).
// The eight fine values of a coarse cell (child c0 + 2 c1 + 4 c2):
// interpconstant, then interplinear in directions 0, 1, 2, each adding
// dxf * slope with dxf = -0.25 or 0.25 (-half + (id + half) / 2, exactly).
// (-0.25) * s is -(0.25 * s) exactly and v + (-q) is v - q, and the partial
// sums after directions 0 and 1 are shared by the children that agree on
// them: the same roundings as adding the three terms child by child, with 3
// products and 14 sums instead of 24 and 24.
__device__ __forceinline__ void childValues(double v, bool lin, double s0, double s1, double s2, double f[8]) {
  if (!lin) {
#pragma unroll
    for (int c = 0; c < 8; ++c) f[c] = v;
    return;
  }
  const double q0 = 0.25 * s0, q1 = 0.25 * s1, q2 = 0.25 * s2;
  const double a[2] = {v - q0, v + q0};
#pragma unroll
  for (int c0 = 0; c0 < 2; ++c0) {
    const double b0 = a[c0] - q1, b1 = a[c0] + q1;
    f[c0] = b0 - q2;
    f[c0 + 4] = b0 + q2;
    f[c0 + 2] = b1 - q2;
    f[c0 + 6] = b1 + q2;
  }
}

template <class FI>
__device__ __forceinline__ void interpCell(const FiBox& b, int I, int J, int K, const double* s, int sy, int sz,
                                           FI fidx, double* __restrict__ fine, int pwc) {
  const double v = s[0];
  const bool lin = !pwc && I >= b.mlo[0] && I <= b.mhi[0] && J >= b.mlo[1] && J <= b.mhi[1] && K >= b.mlo[2] &&
                   K <= b.mhi[2];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  if (lin) {
    s0 = 0.5 * (s[1] - s[-1]);
    s1 = 0.5 * (s[sy] - s[-sy]);
    s2 = 0.5 * (s[sz] - s[-sz]);
    double smax = v, smin = v;
#pragma unroll
    for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const double w = s[di + dj * sy + dk * sz];
          smax = fmax(smax, w);
          smin = fmin(smin, w);
        }
    const double deltasum = 0.5 * (fabs(s0) + fabs(s1) + fabs(s2));
    double eta = fmin(smax - v, v - smin);
    // the reference's 1.e-9 is a single-precision Fortran literal
    if (eta <= (double)1.0e-9f * fabs(smax)) {
      eta = 0.0;
    } else if (deltasum > eta) {
      eta = eta / deltasum;
    } else {
      eta = 1.0;
    }
    s0 = eta * s0;
    s1 = eta * s1;
    s2 = eta * s2;
  }
  double f[8];
  childValues(v, lin, s0, s1, s2, f);
#pragma unroll
  for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
    for (int c1 = 0; c1 < 2; ++c1)
#pragma unroll
      for (int c0 = 0; c0 < 2; ++c0) fine[fidx(b.fbox, 2 * I + c0, 2 * J + c1, 2 * K + c2)] = f[c0 + 2 * c1 + 4 * c2];
}

// One-kernel path: block = fine box.  Its gather items (grow(b, 1) & domain
// split over the coarse boxes, LevelData::copyTo into the coarsened fine
// layout, FineInterp.cpp:148-160) go to shared memory; then each thread takes
// a column segment of b's coarse cells, consecutive threads on consecutive x,
// so each of the eight fine stores of a warp covers contiguous slots.
template <class CI, class FI>
__global__ void __launch_bounds__(kFusedThreads) k_fi_fused(const FiBox* boxes, const int* itemStart,
                                                            const FiGather* gathers, CI cidx,
                                                            const double* __restrict__ coarse, FI fidx,
                                                            double* __restrict__ fine, int pwc) {
  extern __shared__ double st[];
  const FiBox b = boxes[blockIdx.x];
  const int sy = b.sx, sz = b.sx * b.sy;
  // The cells of all items in one enumeration, kLoadILP loads in flight per
  // thread; each thread walks the items forward (its cells only increase).
  const int i1 = itemStart[blockIdx.x + 1];
  int it = itemStart[blockIdx.x];
  for (int base = threadIdx.x; base < b.gcells; base += kLoadILP * kFusedThreads) {
    double v[kLoadILP];
    int at[kLoadILP];
#pragma unroll
    for (int u = 0; u < kLoadILP; ++u) {
      const int q = base + u * kFusedThreads;
      at[u] = -1;
      if (q < b.gcells) {
        while (it + 1 < i1 && gathers[it + 1].cstart <= q) ++it;
        const FiGather& g = gathers[it];
        const int nx = g.hi[0] - g.lo[0] + 1, ny = g.hi[1] - g.lo[1] + 1;
        const int p = q - g.cstart, r = p / nx, k = r / ny;
        const int I = g.lo[0] + (p - r * nx), J = g.lo[1] + (r - k * ny), K = g.lo[2] + k;
        at[u] = (I - b.lo[0] + 1) + sy * (J - b.lo[1] + 1) + sz * (K - b.lo[2] + 1);
        v[u] = coarse[cidx(g.cbox, I, J, K)];
      }
    }
#pragma unroll
    for (int u = 0; u < kLoadILP; ++u)
      if (at[u] >= 0) st[at[u]] = v[u];
  }
  __syncthreads();
  // Work items: a column (i, j) of the coarsened box over up to kSeg planes,
  // consecutive threads on consecutive i.  Down a column the 27-cell extrema
  // come from three plane extrema, each plane's computed once.  Extrema over
  // the same cells are the same numbers in any order; cells outside b_mod
  // (whose neighbours may lie outside the domain) ignore them.
  const auto fr = fidx.rows(b.fbox);
  const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
  const int ncol = nx * ny, nseg = (nz + kSeg - 1) / kSeg;
  for (int w = threadIdx.x; w < ncol * nseg; w += kFusedThreads) {
    const int seg = w / ncol, col = w - seg * ncol;
    const int j = col / nx, i = col - j * nx;
    const int k0 = seg * kSeg, k1 = min(k0 + kSeg, nz);
    const int I = b.lo[0] + i, J = b.lo[1] + j;
    const bool linIJ = !pwc && I >= b.mlo[0] && I <= b.mhi[0] && J >= b.mlo[1] && J <= b.mhi[1];
    const double* c = st + (i + 1) + sy * (j + 1) + sz * (k0 + 1);
    double mxm = 0.0, mnm = 0.0, mx0 = 0.0, mn0 = 0.0;
    if (linIJ) {
      planeExtrema(c - sz, sy, mxm, mnm);
      planeExtrema(c, sy, mx0, mn0);
    }
    int l = fr.lin(i, j, k0);
    for (int k = k0; k < k1; ++k, c += sz, l += 2 * fr.dz) {
      const double v = c[0];
      const int K = b.lo[2] + k;
      const bool lin = linIJ && K >= b.mlo[2] && K <= b.mhi[2];
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      if (linIJ) {
        double mxp, mnp;
        planeExtrema(c + sz, sy, mxp, mnp);
        if (lin) {
          // interpcentralslope, interplimit
          s0 = 0.5 * (c[1] - c[-1]);
          s1 = 0.5 * (c[sy] - c[-sy]);
          s2 = 0.5 * (c[sz] - c[-sz]);
          const double smax = fmax(fmax(mxm, mx0), mxp), smin = fmin(fmin(mnm, mn0), mnp);
          const double deltasum = 0.5 * (fabs(s0) + fabs(s1) + fabs(s2));
          double eta = fmin(smax - v, v - smin);
          // the reference's 1.e-9 is a single-precision Fortran literal
          if (eta <= (double)1.0e-9f * fabs(smax)) {
            eta = 0.0;
          } else if (deltasum > eta) {
            eta = eta / deltasum;
          } else {
            eta = 1.0;
          }
          s0 = eta * s0;
          s1 = eta * s1;
          s2 = eta * s2;
        }
        mxm = mx0;
        mnm = mn0;
        mx0 = mxp;
        mn0 = mnp;
      }
      // interpconstant, then interplinear dir 0, 1, 2
      double f[8];
      childValues(v, lin, s0, s1, s2, f);
#pragma unroll
      for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
        for (int c1 = 0; c1 < 2; ++c1)
#pragma unroll
          for (int c0 = 0; c0 < 2; ++c0)
            fine[fr.at(l + c0 + fr.dy * c1 + fr.dz * c2, (c0 + c1 + c2) & 1)] = f[c0 + 2 * c1 + 4 * c2];
    }
  }
}

// Two-kernel path, step 1: coarse cells of grow(b, 1) & domain into the
// staging blocks in device memory.
template <class CI>
__global__ void k_fi_gather(const FiGather* gathers, const FiBox* boxes, const Chunk* ch, CI cidx,
                            const double* __restrict__ coarse, double* __restrict__ stage) {
  const Chunk c = ch[blockIdx.x];
  const FiGather g = gathers[c.box];
  const int q = c.start + threadIdx.x;
  const int nx = g.hi[0] - g.lo[0] + 1, ny = g.hi[1] - g.lo[1] + 1, nz = g.hi[2] - g.lo[2] + 1;
  if (q >= nx * ny * nz) return;
  const int r = q / nx, k = r / ny;
  const int I = g.lo[0] + (q - r * nx), J = g.lo[1] + (r - k * ny), K = g.lo[2] + k;
  const FiBox& b = boxes[g.fi];
  stage[b.soff + (I - b.lo[0] + 1) + (int64_t)b.sx * ((J - b.lo[1] + 1) + (int64_t)b.sy * (K - b.lo[2] + 1))] =
      coarse[cidx(g.cbox, I, J, K)];
}

// Two-kernel path, step 2: one thread per coarse cell of b.
template <class FI>
__global__ void k_fi_interp(const FiBox* boxes, const Chunk* ch, const double* __restrict__ stage, FI fidx,
                            double* __restrict__ fine, int pwc) {
  const Chunk c = ch[blockIdx.x];
  const FiBox b = boxes[c.box];
  const int q = c.start + threadIdx.x;
  const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
  if (q >= nx * ny * nz) return;
  const int r = q / nx, kk = r / ny;
  const int i = q - r * nx, j = r - kk * ny;
  const int sy = b.sx, sz = b.sx * b.sy;
  interpCell(b, b.lo[0] + i, b.lo[1] + j, b.lo[2] + kk, stage + b.soff + (i + 1) + sy * (j + 1) + sz * (kk + 1),
             sy, sz, fidx, fine, pwc);
}

template <class CI, class FI>
void launch(cudaStream_t s, bool fused, int nbox, size_t smem, int nGatherCh, int nBoxCh, const FiBox* boxes,
            const int* itemStart, const FiGather* gathers, const Chunk* gatherCh, const Chunk* boxCh, double* stage,
            CI cidx, const double* coarse, FI fidx, double* fine, bool pwc) {
  if (fused) {
    if (nbox == 0) return;
    // above the default 48 KB the kernel needs the opt-in, which is per device
    // (set on every such launch: a host call, no device work)
    if (smem > 48 * 1024)
      ck(cudaFuncSetAttribute(k_fi_fused<CI, FI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmemMax),
         "fine interpolation smem attribute");
    k_fi_fused<CI, FI><<<nbox, kFusedThreads, smem, s>>>(boxes, itemStart, gathers, cidx, coarse, fidx, fine,
                                                         pwc ? 1 : 0);
    ck(cudaGetLastError(), "fine interpolation");
    addLaunches(1);
    return;
  }
  if (nGatherCh) {
    k_fi_gather<<<nGatherCh, kChunk, 0, s>>>(gathers, boxes, gatherCh, cidx, coarse, stage);
    ck(cudaGetLastError(), "fine interpolation gather");
    addLaunches(1);
  }
  if (nBoxCh) {
    k_fi_interp<<<nBoxCh, kChunk, 0, s>>>(boxes, boxCh, stage, fidx, fine, pwc ? 1 : 0);
    ck(cudaGetLastError(), "fine interpolation");
    addLaunches(1);
  }
}

}  // namespace

int64_t flatBoxes(const std::vector<Box>& grids, std::vector<FlatBox>& out) {
  out.clear();
  int64_t off = 0;
  for (const Box& b : grids) {
    FlatBox f;
    for (int d = 0; d < 3; ++d) f.lo[d] = b.lo[d];
    f.nx = b.size(0);
    f.ny = b.size(1);
    f.off = off;
    off += b.numPts();
    out.push_back(f);
  }
  return off;
}

FineInterpOp::FineInterpOp(const std::vector<Box>& coarse, const BoxIndex& cindex, const Box& coarseDomain,
                           const std::vector<Box>& fine, cudaStream_t s, bool allowFused)
    : s_(s), own_(s) {
  std::vector<FiBox> boxes;
  std::vector<FiGather> gathers;
  std::vector<Chunk> boxCh, gatherCh;
  std::vector<int> itemStart(1, 0);
  std::vector<int> hits;
  int64_t soff = 0, maxStage = 0;
  for (size_t f = 0; f < fine.size(); ++f) {
    if (!fine[f].coarsenable(2)) throw std::invalid_argument("cmg: fine box not coarsenable by 2");
    const Box b = fine[f].coarsen(2);
    // b_mod for the PCInterp boundary type (FineInterp.cpp:285-292)
    const Box g = b.grow(1) & coarseDomain;
    const Box m = g.grow(-1);
    FiBox fb;
    fb.fbox = (int)f;
    for (int d = 0; d < 3; ++d) {
      fb.lo[d] = b.lo[d];
      fb.hi[d] = b.hi[d];
      fb.mlo[d] = m.lo[d];
      fb.mhi[d] = m.hi[d];
    }
    fb.sx = b.size(0) + 2;
    fb.sy = b.size(1) + 2;
    fb.soff = soff;
    fb.gcells = 0;
    const int64_t stageCells = (int64_t)fb.sx * fb.sy * (b.size(2) + 2);
    soff += stageCells;
    maxStage = std::max(maxStage, stageCells);
    const int item = (int)boxes.size();
    boxes.push_back(fb);
    chunks(boxCh, item, b.numPts());
    fineCells_ += fine[f].numPts();
    cindex.query(coarse, g, hits);
    int64_t inG = 0, inB = 0;
    for (int cb : hits) {
      const Box r = g & coarse[cb];
      if (r.empty()) continue;
      FiGather gg;
      gg.fi = item;
      gg.cbox = cb;
      gg.cstart = (int)inG;
      for (int d = 0; d < 3; ++d) {
        gg.lo[d] = r.lo[d];
        gg.hi[d] = r.hi[d];
      }
      chunks(gatherCh, (int)gathers.size(), r.numPts());
      gathers.push_back(gg);
      inG += r.numPts();
      inB += (b & coarse[cb]).numPts();
    }
    // the cells the items hold (all of grow(b, 1) & domain when nested)
    boxes[item].gcells = (int)inG;
    itemStart.push_back((int)gathers.size());
    if (inG != g.numPts()) nested_ = false;
    if (inB != b.numPts()) covered_ = false;
  }
  nbox_ = (int)boxes.size();
  fused_ = allowFused && (size_t)maxStage * sizeof(double) <= kFusedSmemMax;
  smem_ = (size_t)maxStage * sizeof(double);
  stageCells_ = fused_ ? 0 : soff;
  nBoxCh_ = (int)boxCh.size();
  nGatherCh_ = (int)gatherCh.size();

  // one device allocation, 256-byte aligned parts
  auto up = [](size_t n) { return (n + 255) & ~(size_t)255; };
  const size_t bBytes = up(boxes.size() * sizeof(FiBox)), bcBytes = up(boxCh.size() * sizeof(Chunk));
  const size_t gBytes = up(gathers.size() * sizeof(FiGather)), gcBytes = up(gatherCh.size() * sizeof(Chunk));
  const size_t iBytes = up(itemStart.size() * sizeof(int));
  const size_t sBytes = up((size_t)stageCells_ * sizeof(double));
  const size_t tables = bBytes + bcBytes + gBytes + gcBytes + iBytes;
  if (tables + sBytes == 0) return;
  ck(cudaMallocAsync(&mem_, tables + sBytes, s_), "cudaMalloc fine interpolation plan");
  char* p = (char*)mem_;
  std::vector<char> host(tables);
  auto put = [&](size_t at, const void* src, size_t n) {
    if (n) std::memcpy(host.data() + at, src, n);
  };
  put(0, boxes.data(), boxes.size() * sizeof(FiBox));
  put(bBytes, boxCh.data(), boxCh.size() * sizeof(Chunk));
  put(bBytes + bcBytes, gathers.data(), gathers.size() * sizeof(FiGather));
  put(bBytes + bcBytes + gBytes, gatherCh.data(), gatherCh.size() * sizeof(Chunk));
  put(bBytes + bcBytes + gBytes + gcBytes, itemStart.data(), itemStart.size() * sizeof(int));
  ck(cudaMemcpyAsync(p, host.data(), host.size(), cudaMemcpyHostToDevice, s_), "fine interpolation plan h2d");
  boxes_ = (const FiBox*)p;
  boxCh_ = (const Chunk*)(p + bBytes);
  gathers_ = (const FiGather*)(p + bBytes + bcBytes);
  gatherCh_ = (const Chunk*)(p + bBytes + bcBytes + gBytes);
  itemStart_ = (const int*)(p + bBytes + bcBytes + gBytes + gcBytes);
  stage_ = stageCells_ ? (double*)(p + tables) : nullptr;
  ck(cudaStreamSynchronize(s_), "fine interpolation plan sync");
}

FineInterpOp::~FineInterpOp() {
  if (mem_) {
    cudaStreamSynchronize(s_);
    cudaFreeAsync(mem_, own_);
    cudaStreamSynchronize(own_);
  }
}

void FineInterpOp::check(bool pwc) const {
  if (pwc ? !covered_ : !nested_)
    throw std::invalid_argument(pwc ? "cmg: coarsened fine boxes not covered by the coarse level"
                                    : "cmg: fine level not properly nested in the coarse level");
}

void FineInterpOp::run(const BoxDesc* cboxes, const double* coarse, const BoxDesc* fboxes, double* fine, bool pwc) {
  check(pwc);
  launch(s_, fused_, nbox_, smem_, nGatherCh_, nBoxCh_, boxes_, itemStart_, gathers_, gatherCh_, boxCh_, stage_,
         RBCells{cboxes}, coarse, RBCells{fboxes}, fine, pwc);
}

void FineInterpOp::runFlat(const FlatBox* cboxes, const double* coarse, const FlatBox* fboxes, double* fine,
                           bool pwc) {
  check(pwc);
  launch(s_, fused_, nbox_, smem_, nGatherCh_, nBoxCh_, boxes_, itemStart_, gathers_, gatherCh_, boxCh_, stage_,
         FlatCells{cboxes}, coarse, FlatCells{fboxes}, fine, pwc);
}

}  // namespace cmg
