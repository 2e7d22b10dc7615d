// FineInterp on the device (fineinterp.H).  Bit-exact with the reference:
// compiled with --fmad=false, every slope, limiter and fine value is formed
// with the reference's operations in its order (InterpF.ChF:48-71, 135-312,
// 318-369).
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "fineinterp.H"
#include "kernels.H"

namespace cmg {

namespace {

constexpr int kChunk = 256;

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

// Element index of cell (i, j, k) of box `box` in a red-black level field.
struct RBCells {
  const BoxDesc* b;
  __device__ __forceinline__ int64_t operator()(int box, int i, int j, int k) const {
    return cellIndex(b[box], i, j, k);
  }
};

// ... in a flat valid-cell array.
struct FlatCells {
  const FlatBox* b;
  __device__ __forceinline__ int64_t operator()(int box, int i, int j, int k) const {
    const FlatBox& x = b[box];
    return x.off + (i - x.lo[0]) + (int64_t)x.nx * ((j - x.lo[1]) + (int64_t)x.ny * (k - x.lo[2]));
  }
};

// Coarse cells of grow(b, 1) & domain into the staging blocks
// (LevelData::copyTo into the coarsened fine layout, FineInterp.cpp:148-160).
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

// One thread per coarse cell of b: interpconstant, then on b_mod the central
// slopes (interpcentralslope), the limiter (interplimit) and the three
// linear corrections (interplinear, dir 0, 1, 2).  Threads of a warp take
// consecutive x cells, so each of the eight fine stores covers contiguous
// slots of one colour half.
template <class FI>
__global__ void k_fi_interp(const FiBox* boxes, const Chunk* ch, const double* __restrict__ stage, FI fidx,
                            double* __restrict__ fine, int pwc) {
  const Chunk c = ch[blockIdx.x];
  const FiBox b = boxes[c.box];
  const int q = c.start + threadIdx.x;
  const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
  if (q >= nx * ny * nz) return;
  const int r = q / nx, kk = r / ny;
  const int I = b.lo[0] + (q - r * nx), J = b.lo[1] + (r - kk * ny), K = b.lo[2] + kk;
  const int64_t sy = b.sx, sz = (int64_t)b.sx * b.sy;
  const double* s = stage + b.soff + (I - b.lo[0] + 1) + sy * (J - b.lo[1] + 1) + sz * (K - b.lo[2] + 1);
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
#pragma unroll
  for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
    for (int c1 = 0; c1 < 2; ++c1)
#pragma unroll
      for (int c0 = 0; c0 < 2; ++c0) {
        double f = v;
        if (lin) {
          // dxf = -half + (id + half) / 2: -0.25 or 0.25, exactly
          f = f + (c0 ? 0.25 : -0.25) * s0;
          f = f + (c1 ? 0.25 : -0.25) * s1;
          f = f + (c2 ? 0.25 : -0.25) * s2;
        }
        fine[fidx(b.fbox, 2 * I + c0, 2 * J + c1, 2 * K + c2)] = f;
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
                           const std::vector<Box>& fine, cudaStream_t s)
    : s_(s) {
  std::vector<FiBox> boxes;
  std::vector<FiGather> gathers;
  std::vector<Chunk> boxCh, gatherCh;
  std::vector<int> hits;
  int64_t soff = 0;
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
    soff += (int64_t)fb.sx * fb.sy * (b.size(2) + 2);
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
      for (int d = 0; d < 3; ++d) {
        gg.lo[d] = r.lo[d];
        gg.hi[d] = r.hi[d];
      }
      chunks(gatherCh, (int)gathers.size(), r.numPts());
      gathers.push_back(gg);
      inG += r.numPts();
      inB += (b & coarse[cb]).numPts();
    }
    if (inG != g.numPts()) nested_ = false;
    if (inB != b.numPts()) covered_ = false;
  }
  stageCells_ = soff;
  nBoxCh_ = (int)boxCh.size();
  nGatherCh_ = (int)gatherCh.size();

  // one device allocation, 256-byte aligned parts
  auto up = [](size_t n) { return (n + 255) & ~(size_t)255; };
  const size_t bBytes = up(boxes.size() * sizeof(FiBox)), bcBytes = up(boxCh.size() * sizeof(Chunk));
  const size_t gBytes = up(gathers.size() * sizeof(FiGather)), gcBytes = up(gatherCh.size() * sizeof(Chunk));
  const size_t sBytes = up((size_t)stageCells_ * sizeof(double));
  const size_t total = bBytes + bcBytes + gBytes + gcBytes + sBytes;
  if (total == 0) return;
  ck(cudaMallocAsync(&mem_, total, s_), "cudaMalloc fine interpolation plan");
  char* p = (char*)mem_;
  std::vector<char> host(bBytes + bcBytes + gBytes + gcBytes);
  auto put = [&](size_t at, const void* src, size_t n) {
    if (n) std::memcpy(host.data() + at, src, n);
  };
  put(0, boxes.data(), boxes.size() * sizeof(FiBox));
  put(bBytes, boxCh.data(), boxCh.size() * sizeof(Chunk));
  put(bBytes + bcBytes, gathers.data(), gathers.size() * sizeof(FiGather));
  put(bBytes + bcBytes + gBytes, gatherCh.data(), gatherCh.size() * sizeof(Chunk));
  if (!host.empty()) ck(cudaMemcpyAsync(p, host.data(), host.size(), cudaMemcpyHostToDevice, s_), "fine interpolation plan h2d");
  boxes_ = (const FiBox*)p;
  boxCh_ = (const Chunk*)(p + bBytes);
  gathers_ = (const FiGather*)(p + bBytes + bcBytes);
  gatherCh_ = (const Chunk*)(p + bBytes + bcBytes + gBytes);
  stage_ = (double*)(p + bBytes + bcBytes + gBytes + gcBytes);
  ck(cudaStreamSynchronize(s_), "fine interpolation plan sync");
}

FineInterpOp::~FineInterpOp() {
  if (mem_) {
    cudaFreeAsync(mem_, s_);
    cudaStreamSynchronize(s_);
  }
}

void FineInterpOp::check(bool pwc) const {
  if (pwc ? !covered_ : !nested_)
    throw std::invalid_argument(pwc ? "cmg: coarsened fine boxes not covered by the coarse level"
                                    : "cmg: fine level not properly nested in the coarse level");
}

void FineInterpOp::run(const BoxDesc* cboxes, const double* coarse, const BoxDesc* fboxes, double* fine, bool pwc) {
  check(pwc);
  if (nGatherCh_) {
    k_fi_gather<<<nGatherCh_, kChunk, 0, s_>>>(gathers_, boxes_, gatherCh_, RBCells{cboxes}, coarse, stage_);
    ck(cudaGetLastError(), "fine interpolation gather");
  }
  if (nBoxCh_) {
    k_fi_interp<<<nBoxCh_, kChunk, 0, s_>>>(boxes_, boxCh_, stage_, RBCells{fboxes}, fine, pwc ? 1 : 0);
    ck(cudaGetLastError(), "fine interpolation");
  }
  addLaunches(kernelLaunches());
}

void FineInterpOp::runFlat(const FlatBox* cboxes, const double* coarse, const FlatBox* fboxes, double* fine,
                           bool pwc) {
  check(pwc);
  if (nGatherCh_) {
    k_fi_gather<<<nGatherCh_, kChunk, 0, s_>>>(gathers_, boxes_, gatherCh_, FlatCells{cboxes}, coarse, stage_);
    ck(cudaGetLastError(), "fine interpolation gather");
  }
  if (nBoxCh_) {
    k_fi_interp<<<nBoxCh_, kChunk, 0, s_>>>(boxes_, boxCh_, stage_, FlatCells{fboxes}, fine, pwc ? 1 : 0);
    ck(cudaGetLastError(), "fine interpolation");
  }
  addLaunches(kernelLaunches());
}

}  // namespace cmg
