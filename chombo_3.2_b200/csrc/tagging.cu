// Device-side tagging (see tagging.H).
#include "tagging.H"

#include <algorithm>
#include <stdexcept>
#include <string>

#include "synthdev.H"

namespace cmg {

namespace {

struct TagBox {
  int lo[3], n[3];
  int64_t off;  // first value of the box in the per-cell array (x fastest)
};
struct TagChunk {
  int box, start;  // 256 cells of one box
};
enum { TAG_THREADS = 256 };

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("cmg: tagging ") + what + ": " + cudaGetErrorString(e));
}

// |rhs| at every cell centre of the level's boxes, and its maximum.  The
// maximum of non-negative doubles is taken on their bit patterns, which order
// the same way.
__global__ void __launch_bounds__(TAG_THREADS) k_tag_eval(const TagBox* __restrict__ boxes,
                                                         const TagChunk* __restrict__ chunks, double dx,
                                                         cmg_synth::Bumps bumps, double* vals,
                                                         unsigned long long* dMax) {
  const TagChunk ch = chunks[blockIdx.x];
  const TagBox b = boxes[ch.box];
  const int q = ch.start + threadIdx.x;
  double a = 0.0;
  if (q < b.n[0] * b.n[1] * b.n[2]) {
    const int i = b.lo[0] + q % b.n[0], j = b.lo[1] + (q / b.n[0]) % b.n[1], k = b.lo[2] + q / (b.n[0] * b.n[1]);
    a = fabs(devBumps(bumps, (i + 0.5) * dx, (j + 0.5) * dx, (k + 0.5) * dx));
    vals[b.off + q] = a;
  }
  unsigned long long m = (unsigned long long)__double_as_longlong(a);
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  __shared__ unsigned long long wmax[TAG_THREADS / 32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < TAG_THREADS / 32; ++w) m = wmax[w] > m ? wmax[w] : m;
    atomicMax(dMax, m);
  }
}

// Tag map of the domain (one byte per cell, x fastest): cells with
// |rhs| > thresh * max|rhs|.
__global__ void __launch_bounds__(TAG_THREADS) k_tag_mark(const TagBox* __restrict__ boxes,
                                                         const TagChunk* __restrict__ chunks,
                                                         const double* __restrict__ vals,
                                                         const unsigned long long* dMax, double thresh, int dlo0,
                                                         int dlo1, int dlo2, int64_t dn0, int64_t dn1,
                                                         uint8_t* map) {
  const TagChunk ch = chunks[blockIdx.x];
  const TagBox b = boxes[ch.box];
  const int q = ch.start + threadIdx.x;
  if (q >= b.n[0] * b.n[1] * b.n[2]) return;
  const double tagVal = __longlong_as_double((long long)*dMax) * thresh;
  if (!(vals[b.off + q] > tagVal)) return;
  const int i = b.lo[0] + q % b.n[0], j = b.lo[1] + (q / b.n[0]) % b.n[1], k = b.lo[2] + q / (b.n[0] * b.n[1]);
  map[(i - dlo0) + dn0 * ((j - dlo1) + dn1 * (int64_t)(k - dlo2))] = 1;
}

// One-cell growth along one axis, clipped to the domain: three passes give
// the growth of every tag by the 3x3x3 box.
__global__ void k_tag_grow(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int64_t n0, int64_t n1,
                           int64_t n2, int axis) {
  const int64_t total = n0 * n1 * n2;
  const int64_t stride = axis == 0 ? 1 : axis == 1 ? n0 : n0 * n1;
  const int64_t ext = axis == 0 ? n0 : axis == 1 ? n1 : n2;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = (q / stride) % ext;
    uint8_t v = in[q];
    if (c > 0) v |= in[q - stride];
    if (c + 1 < ext) v |= in[q + stride];
    out[q] = v;
  }
}

}  // namespace

DeviceTagger::DeviceTagger(cudaStream_t s) : s_(s) {}

namespace {
void release(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}
void grow(void** p, size_t bytes, cudaStream_t s) {
  if (*p) ck(cudaFreeAsync(*p, s), "free");
  *p = nullptr;
  ck(cudaMallocAsync(p, bytes, s), "alloc");
}
}  // namespace

DeviceTagger::~DeviceTagger() {
  release(cells_, s_);
  release(vals_, s_);
  release(map_[0], s_);
  release(map_[1], s_);
  release(dMax_, s_);
  cudaStreamSynchronize(s_);
}

void DeviceTagger::tags(const std::vector<Box>& grids, const Box& domain, double dx, const cmg_synth::Bumps& bumps,
                        double thresh, CellSet& out) {
  std::vector<TagBox> tb;
  std::vector<TagChunk> tc;
  int64_t n = 0;
  for (size_t b = 0; b < grids.size(); ++b) {
    const Box& g = grids[b];
    if (g.empty()) continue;
    TagBox t;
    for (int d = 0; d < 3; ++d) {
      t.lo[d] = g.lo[d];
      t.n[d] = g.size(d);
    }
    t.off = n;
    const int64_t cells = g.numPts();
    if (cells >= (int64_t)1 << 31) throw std::invalid_argument("cmg: box too large to tag");
    for (int64_t s = 0; s < cells; s += TAG_THREADS) tc.push_back(TagChunk{(int)tb.size(), (int)s});
    tb.push_back(t);
    n += cells;
  }
  out.define(domain, false);
  if (n == 0 || domain.empty()) return;
  if (tc.size() > 0x7fffffffu) throw std::invalid_argument("cmg: level too large to tag");
  const size_t tableBytes = tb.size() * sizeof(TagBox) + tc.size() * sizeof(TagChunk);
  if (tableBytes > cellsBytes_) {
    grow(&cells_, tableBytes, s_);
    cellsBytes_ = tableBytes;
  }
  if ((size_t)n > valsCount_) {
    grow((void**)&vals_, n * sizeof(double), s_);
    valsCount_ = n;
  }
  const size_t mapBytes = (size_t)domain.numPts();
  if (mapBytes > mapBytes_) {
    for (auto& m : map_) grow((void**)&m, mapBytes, s_);
    mapBytes_ = mapBytes;
  }
  if (!dMax_) grow((void**)&dMax_, sizeof(unsigned long long), s_);
  TagBox* dBoxes = (TagBox*)cells_;
  TagChunk* dChunks = (TagChunk*)((char*)cells_ + tb.size() * sizeof(TagBox));
  ck(cudaMemcpyAsync(dBoxes, tb.data(), tb.size() * sizeof(TagBox), cudaMemcpyHostToDevice, s_), "copy");
  ck(cudaMemcpyAsync(dChunks, tc.data(), tc.size() * sizeof(TagChunk), cudaMemcpyHostToDevice, s_), "copy");
  ck(cudaMemsetAsync(dMax_, 0, sizeof(unsigned long long), s_), "memset");
  ck(cudaMemsetAsync(map_[0], 0, mapBytes, s_), "memset");
  k_tag_eval<<<(unsigned)tc.size(), TAG_THREADS, 0, s_>>>(dBoxes, dChunks, dx, bumps, vals_, dMax_);
  const int64_t dn0 = domain.size(0), dn1 = domain.size(1), dn2 = domain.size(2);
  k_tag_mark<<<(unsigned)tc.size(), TAG_THREADS, 0, s_>>>(dBoxes, dChunks, vals_, dMax_, thresh, domain.lo[0],
                                                         domain.lo[1], domain.lo[2], dn0, dn1, map_[0]);
  const int grid = (int)std::min<int64_t>(((int64_t)mapBytes + 255) / 256, 148 * 16);
  for (int axis = 0; axis < 3; ++axis)
    k_tag_grow<<<grid, 256, 0, s_>>>(map_[axis & 1], map_[(axis + 1) & 1], dn0, dn1, dn2, axis);
  ck(cudaGetLastError(), "launch");
  ck(cudaMemcpyAsync(out.bits.data(), map_[1], mapBytes, cudaMemcpyDeviceToHost, s_), "copy back");
  ck(cudaStreamSynchronize(s_), "sync");
}

}  // namespace cmg
