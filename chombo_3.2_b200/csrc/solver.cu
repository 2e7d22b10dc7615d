// GPU AMR multigrid solver.  The V-cycle control flow restates
// AMRMultiGrid::solveNoInitResid / AMRVCycle / computeAMRResidual
// (AMRElliptic/AMRMultiGrid.H:682-1124, 1341-1419) and MultiGrid::cycle
// (AMRElliptic/MultiGrid.H:629-696); every step below names the operator
// method it performs.
#include "solver.H"
#include "fineinterp.H"
#include "hostpool.H"

#include <cstdint>
#include <algorithm>
#include <chrono>
#include <mutex>
#include <exception>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace cmg {

namespace {

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "cmg: %s: %s", what, cudaGetErrorString(e));
    throw std::runtime_error(buf);
  }
}

// Valid (or face) region of box b for the user data layout.
Box userRegion(const Box& b, int faceDir) {
  Box r = b;
  if (faceDir >= 0) r.hi[faceDir] += 1;
  return r;
}

struct RegionCopy {
  int box;
  int lo[3], hi[3];
  int64_t srcOff;
};

__global__ void k_scatter(const BoxDesc* boxes, const RegionCopy* rc, double* dev, const double* src, int toDev) {
  const RegionCopy r = rc[blockIdx.x];
  const BoxDesc b = boxes[r.box];
  int nx = r.hi[0] - r.lo[0] + 1, ny = r.hi[1] - r.lo[1] + 1, nz = r.hi[2] - r.lo[2] + 1;
  for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
    int i = r.lo[0] + q % nx, t = q / nx, j = r.lo[1] + t % ny, k = r.lo[2] + t / ny;
    int64_t c = cellIndex(b, i, j, k);
    if (toDev)
      dev[c] = src[r.srcOff + q];
    else
      const_cast<double*>(src)[r.srcOff + q] = dev[c];
  }
}

}  // namespace

namespace {
// Keep freed blocks in the stream-ordered pool of each device for reuse by
// the next hierarchy instead of returning them to the driver.
void keepPoolMemory() {
  static std::once_flag once[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::call_once(once[dev], [dev]() {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  });
}
}  // namespace

DevBuf::DevBuf(size_t n, cudaStream_t stream) : bytes(n), s(stream) {
  keepPoolMemory();
  ck(cudaMallocAsync(&p, n ? n : 1, s), "cudaMalloc");
}
DevBuf::~DevBuf() {
  if (p) cudaFreeAsync(p, s);
}

// Work moves to the caller's stream; allocations stay on the hierarchy's own
// stream (so they can be freed whatever becomes of the caller's), each one
// completed before the work stream can use it.
void Solver::setStream(cudaStream_t s) {
  if (!s) s = own_;
  if (s == s_) return;
  ck(cudaStreamSynchronize(s_), "stream switch");
  s_ = s;
}

void Solver::ownSync() {
  if (s_ != own_) ck(cudaStreamSynchronize(own_), "allocation sync");
}

size_t Solver::deviceBytes() const {
  size_t n = stage_ ? stage_->bytes : 0;
  for (const auto& b : bufs_) n += b->bytes;
  return n;
}

double* Solver::alloc(size_t n) {
  bufs_.emplace_back(new DevBuf(n * sizeof(double), own_));
  ownSync();
  double* p = (double*)bufs_.back()->p;
  ck(cudaMemsetAsync(p, 0, n * sizeof(double), s_), "memset");
  return p;
}

template <class V>
static const typename V::value_type* upload(std::vector<std::unique_ptr<DevBuf>>& bufs, const V& v, cudaStream_t s) {
  if (v.empty()) return nullptr;
  size_t n = v.size() * sizeof(typename V::value_type);
  bufs.emplace_back(new DevBuf(n, s));
  ck(cudaMemcpyAsync(bufs.back()->p, v.data(), n, cudaMemcpyHostToDevice, s), "upload");
  return (const typename V::value_type*)bufs.back()->p;
}

void Solver::uploadLevel(const LevelPlan& p, LevelDev& d) {
  d.boxes = upload(bufs_, p.boxes, s_);
  d.nbox = (int)p.boxes.size();
  d.nelem = p.nelem;
  auto devTasks = [&](const std::vector<GhostTask>& v) {
    std::vector<GhostTaskDev> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
      const GhostTask& t = v[i];
      GhostTaskDev& o = out[i];
      o.dst = p.boxes[t.dst];
      o.src = p.boxes[t.src];
      for (int k = 0; k < 3; ++k) o.shift[k] = t.shift[k];
      o.kind = t.kind;
      o.dir = t.dir;
      o.side = t.side;
      for (int k = 0; k < 3; ++k) {
        o.lo[k] = t.lo[k];
        o.hi[k] = t.hi[k];
      }
      o.ax = parityAxis(t.lo, t.hi);
    }
    return out;
  };
  d.ghost = upload(bufs_, devTasks(p.ghost), s_);
  d.nExchBC = p.nExchBC;
  d.nGhost = (int)p.ghost.size();
  d.ghostStart = upload(bufs_, p.ghostStart, s_);
  d.ghostBlock = upload(bufs_, p.ghostBlock, s_);
  d.slotStart = upload(bufs_, p.slotStart, s_);
  d.slotBlock = upload(bufs_, p.slotBlock, s_);
  d.nSlotsExchBC = p.slotStart.empty() ? 0 : p.slotStart[p.nExchBC];
  d.nSlotsGhost = p.slotStart.empty() ? 0 : p.slotStart.back();
  d.nCellsExchBC = p.ghostStart.empty() ? 0 : p.ghostStart[p.nExchBC];
  d.nCellsGhost = p.ghostStart.empty() ? 0 : p.ghostStart.back();
  d.zero = upload(bufs_, devTasks(p.zeroCovered), s_);
  d.gcells = upload(bufs_, p.gcells, s_);
  d.faceRules = upload(bufs_, p.faceRules, s_);
  d.faceOff = upload(bufs_, p.faceOff, s_);
  d.deferred = upload(bufs_, p.deferred, s_);
  for (int c = 0; c < 2; ++c) {
    d.chGhost[c] = upload(bufs_, p.chunkGhost[c], s_);
    d.chGhostStart[c] = upload(bufs_, p.chunkGhostStart[c], s_);
  }
  d.nDeferred = (int)p.deferred.size();
  for (int c = 0; c < 2; ++c) {
    d.gcStart[c] = p.gcStart[c];
    d.gcExch[c] = p.gcExch[c];
    d.gcCF[c] = p.gcCF[c];
  }
  d.nZero = (int)p.zeroCovered.size();
  d.zeroStart = upload(bufs_, p.zeroStart, s_);
  d.zeroBlock = upload(bufs_, p.zeroBlock, s_);
  d.nCellsZero = p.zeroStart.empty() ? 0 : p.zeroStart.back();
  d.chAll = upload(bufs_, p.chunksAll, s_);
  d.nAll = (int)p.chunksAll.size();
  for (int c = 0; c < 2; ++c) {
    d.chColor[c] = upload(bufs_, p.chunksColor[c], s_);
    d.nColor[c] = (int)p.chunksColor[c].size();
  }
  d.cfC = upload(bufs_, p.cfCoarse, s_);
  d.nCfC = (int)p.cfCoarse.size();
  if (d.nCfC > 0) d.cfTmp = alloc(6 * (size_t)d.nCfC);
  d.cfF = upload(bufs_, p.cfFine, s_);
  d.nCfF = (int)p.cfFine.size();
  d.cfW = upload(bufs_, p.cfW, s_);
  d.cfOff = upload(bufs_, p.cfOff, s_);
  d.items = upload(bufs_, p.toCoarse, s_);
  d.itemChC = upload(bufs_, p.toCoarseChunksC, s_);
  d.nItemChC = (int)p.toCoarseChunksC.size();
  d.itemChF = upload(bufs_, p.toCoarseChunksF, s_);
  d.nItemChF = (int)p.toCoarseChunksF.size();
  d.rfCells = upload(bufs_, p.rfCells, s_);
  d.nRf = (int)p.rfCells.size();
  d.rfC = upload(bufs_, p.rfCoarse, s_);
  d.rfF = upload(bufs_, p.rfFine, s_);
  d.dx = p.dx;
  d.dxCrse = p.dxCrse;
  d.boxHier = upload(bufs_, p.boxHier, s_);
  d.hierStart = upload(bufs_, p.hierStart, s_);
  d.nh = p.hierStart.empty() ? 1 : (int)p.hierStart.size() - 1;
}

// Host plans of one hierarchy: its AMR levels, the multigrid depths below
// level 0 and the plans between consecutive AMR levels.
static void hierarchyPlans(const HierarchyDesc& desc, std::vector<LevelPlan>& amr, std::vector<LevelPlan>& mg) {
  const int nlev = (int)desc.boxes.size();
  if (nlev < 1) throw std::runtime_error("cmg: hierarchy needs at least one level");
  if (nlev > 1 && (desc.periodic[0] || desc.periodic[1] || desc.periodic[2]))
    throw std::invalid_argument("cmg: periodic domains are supported on one-level hierarchies");
  amr.resize(nlev);
  // Host plans, one thread per level and then one per level pair (each pair
  // writes distinct members of its two levels).
  std::vector<Box> doms(nlev);
  std::vector<double> dxs(nlev);
  doms[0] = desc.domain;
  dxs[0] = desc.dx0;
  for (int l = 1; l < nlev; ++l) {
    doms[l] = doms[l - 1].refine(2);
    dxs[l] = dxs[l - 1] / 2;  // m_dx[i] = m_dx[i-1] / refRatio (VCAMRPoissonOp2.cpp:905-912)
  }
  // Multigrid depths of level 0 (AMRPoissonOpFactory::MGnewOp,
  // AMRElliptic/AMRPoissonOp.cpp:1923-1989: exists while the boxes are
  // coarsenable by coarsening * s_maxCoarse(2)).
  const Layout g0(desc.boxes[0]);
  std::vector<int> mgc;
  for (int c = 2; g0.coarsenable(c * 2); c *= 2) mgc.push_back(c);
  mg.resize(mgc.size());
  // Levels and multigrid depths, then the coarse-fine tables of each level
  // pair, as items of the host pool (each item loops over its boxes on the
  // same pool).
  hostParallel(nlev + mgc.size(), [&](size_t i) {
    if (i < (size_t)nlev) {
      const int l = (int)i;
      buildLevel(amr[l], Layout(desc.boxes[l]), doms[l], dxs[l], l > 0 ? dxs[l - 1] : 0.0, desc.bc, desc.periodic);
    } else {
      const int c = mgc[i - nlev];
      buildLevel(mg[i - nlev], g0.coarsen(c), desc.domain.coarsen(c), desc.dx0 * c, 0.0, desc.bc, desc.periodic);
    }
  });
  hostParallel(nlev > 1 ? nlev - 1 : 0, [&](size_t i) {
    const int l = (int)i + 1;
    buildQuadCF(amr[l], amr[l - 1]);
    buildCoarseFine(amr[l], amr[l - 1]);
    buildReflux(amr[l - 1], amr[l], desc.vc != 0);
  });
}

Solver::Solver(const HierarchyDesc& desc, cudaStream_t stream)
    : s_(stream), own_(stream), desc_(desc), alpha0_(desc.alpha), beta0_(desc.beta) {
  const auto t0 = std::chrono::steady_clock::now();
  hierarchyPlans(desc, amr_, mg_);
  std::vector<BottomPlan> bps(1);
  buildBottom(mg_.empty() ? amr_[0] : mg_.back(), bps[0]);
  const auto t1 = std::chrono::steady_clock::now();
  setup(bps);
  planSeconds_ = std::chrono::duration<double>(t1 - t0).count();
  deviceSeconds_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
}

// A forest: hierarchies with the same domain, cell size, level count,
// operator and boundary types (and so the same multigrid depths when their
// level-0 layouts coarsen alike) planned one by one and merged level by level
// (mergeLevels).  Each keeps its own bottom solve; the solve loop keeps a
// residual norm, a stopping rule and an iteration count per hierarchy.
Solver::Solver(const std::vector<HierarchyDesc>& descs, cudaStream_t stream)
    : s_(stream), own_(stream), desc_(descs.at(0)), alpha0_(descs[0].alpha), beta0_(descs[0].beta) {
  const size_t K = descs.size();
  const HierarchyDesc& d0 = descs[0];
  for (const HierarchyDesc& d : descs) {
    bool same = d.domain.lo == d0.domain.lo && d.domain.hi == d0.domain.hi && d.dx0 == d0.dx0 &&
                d.boxes.size() == d0.boxes.size() && d.vc == d0.vc && d.alpha == d0.alpha && d.beta == d0.beta;
    for (int f = 0; f < 6; ++f) same = same && d.bc[f] == d0.bc[f];
    for (int k = 0; k < 3; ++k) same = same && d.periodic[k] == d0.periodic[k];
    if (!same)
      throw std::invalid_argument("cmg: the hierarchies of a forest need the same domain, dx, level count, operator "
                                  "and boundary types");
  }
  std::vector<std::vector<LevelPlan>> amrP(K), mgP(K);
  hostParallel(K, [&](size_t k) { hierarchyPlans(descs[k], amrP[k], mgP[k]); });
  const size_t nlev = amrP[0].size(), nd = mgP[0].size();
  for (size_t k = 0; k < K; ++k)
    if (mgP[k].size() != nd)
      throw std::invalid_argument("cmg: the hierarchies of a forest need the same multigrid depths (level-0 boxes "
                                  "that coarsen alike)");
  // element and box offsets of every part, level by level
  auto offsets = [&](const std::vector<std::vector<LevelPlan>>& P, size_t l, std::vector<int64_t>& eo,
                     std::vector<int>& bo) {
    eo.assign(K, 0);
    bo.assign(K, 0);
    int64_t e = 0;
    int b = 0;
    for (size_t k = 0; k < K; ++k) {
      eo[k] = e;
      bo[k] = b;
      e += P[k][l].nelem;
      b += (int)P[k][l].boxes.size();
    }
  };
  std::vector<std::vector<int64_t>> eoA(nlev), eoM(nd);
  std::vector<std::vector<int>> boA(nlev), boM(nd);
  for (size_t l = 0; l < nlev; ++l) offsets(amrP, l, eoA[l], boA[l]);
  for (size_t d = 0; d < nd; ++d) offsets(mgP, d, eoM[d], boM[d]);
  amr_.resize(nlev);
  mg_.resize(nd);
  for (size_t l = 0; l < nlev; ++l) {
    std::vector<const LevelPlan*> parts;
    for (size_t k = 0; k < K; ++k) parts.push_back(&amrP[k][l]);
    mergeLevels(parts, eoA[l], boA[l], l > 0 ? &eoA[l - 1] : nullptr, l > 0 ? &boA[l - 1] : nullptr,
                l + 1 < nlev ? &eoA[l + 1] : nullptr, amr_[l]);
    desc_.boxes[l] = amr_[l].grids.boxes;
  }
  for (size_t d = 0; d < nd; ++d) {
    std::vector<const LevelPlan*> parts;
    for (size_t k = 0; k < K; ++k) parts.push_back(&mgP[k][d]);
    mergeLevels(parts, eoM[d], boM[d], nullptr, nullptr, nullptr, mg_[d]);
  }
  // each hierarchy's bottom level, its slots moved to the merged elements
  std::vector<BottomPlan> bps(K);
  for (size_t k = 0; k < K; ++k) {
    buildBottom(nd == 0 ? amrP[k][0] : mgP[k][nd - 1], bps[k]);
    const int64_t eo = nd == 0 ? eoA[0][k] : eoM[nd - 1][k];
    for (int& f : bps[k].fab) f += (int)eo;
  }
  setup(bps);
}

void Solver::setup(const std::vector<BottomPlan>& bps) {
  const HierarchyDesc& desc = desc_;
  const int nlev = (int)amr_.size();
  nh_ = (int)bps.size();
  bottomCells_ = desc.domain.numPts();
  for (size_t d = 0; d < mg_.size(); ++d) bottomCells_ /= 8;

  amrDev_.resize(nlev);
  lev_.resize(nlev);
  for (int l = 0; l < nlev; ++l) {
    uploadLevel(amr_[l], amrDev_[l]);
    size_t n = amr_[l].nelem;
    LevelFields& f = lev_[l];
    f.phi = alloc(n);
    f.rhs = alloc(n);
    f.ures = alloc(n);
    f.ucorr = alloc(n);
    f.corr = alloc(n);
    f.res = alloc(n);
    if (desc.vc) {
      f.a = alloc(n);
      for (int d = 0; d < 3; ++d) f.b[d] = alloc(n);
      f.lambda = alloc(n);
    }
  }
  mgDev_.resize(mg_.size());
  mgf_.resize(mg_.size());
  for (size_t d = 0; d < mg_.size(); ++d) {
    uploadLevel(mg_[d], mgDev_[d]);
    size_t n = mg_[d].nelem;
    mgf_[d].corr = alloc(n);
    mgf_[d].res = alloc(n);
    if (desc.vc) {
      mgf_[d].a = alloc(n);
      for (int k = 0; k < 3; ++k) mgf_[d].b[k] = alloc(n);
      mgf_[d].lambda = alloc(n);
    }
  }
  // Bottom solves in the compact slot space of the deepest level, one per
  // hierarchy.
  bottoms_.resize(bps.size());
  maxBottomBoxes_ = 1;
  for (size_t k = 0; k < bps.size(); ++k) {
    const BottomPlan& bp = bps[k];
    BottomWork& w = bottoms_[k];
    const size_t nc = (size_t)bp.nv + bp.ng;
    w.nv = bp.nv;
    w.ng = bp.ng;
    w.nbox = (int)bp.boxStart.size() - 1;
    for (int b = 0; b < w.nbox; ++b) w.maxBoxCells = std::max(w.maxBoxCells, bp.boxStart[b + 1] - bp.boxStart[b]);
    maxBottomBoxes_ = std::max(maxBottomBoxes_, w.nbox);
    w.fab = upload(bufs_, bp.fab, s_);
    w.nb = upload(bufs_, bp.nb, s_);
    for (int c = 0; c < 2; ++c) {
      w.col[c] = upload(bufs_, bp.color[c], s_);
      w.ncol[c] = (int)bp.color[c].size();
    }
    w.boxStart = upload(bufs_, bp.boxStart, s_);
    w.nbv = upload(bufs_, bp.nbv, s_);
    for (int q = 0; q < 10; ++q) w.v[q] = alloc(nc);
    if (desc.vc) {
      w.a = alloc(nc);
      for (int d = 0; d < 3; ++d) w.b[d] = alloc(nc);
      w.lam = alloc(nc);
    }
    bufs_.emplace_back(new DevBuf(4 * sizeof(int), s_));
    w.status = (int*)bufs_.back()->p;
  }
  dBottoms_ = upload(bufs_, bottoms_, s_);
  setBottomGrid(-1);
  dNorm_ = alloc(nh_);
  dMetric_ = alloc(nh_);
  if (nh_ > 1) dEps_ = alloc(nh_);
  bufs_.emplace_back(new DevBuf(nh_ * sizeof(int), s_));
  dActive_ = (int*)bufs_.back()->p;
  ck(cudaMallocHost((void**)&hostScalars_, (2 + 3 * nh_) * sizeof(double)), "pinned scalars");
  ck(cudaMallocHost((void**)&hostActive_, nh_ * sizeof(int)), "pinned flags");
  if (desc.vc) {
    hostA_.resize(nlev);
    for (int d = 0; d < 3; ++d) hostB_[d].resize(nlev);
  }
  ck(cudaStreamSynchronize(s_), "setup");
}

Solver::~Solver() {
  cudaStreamSynchronize(s_);
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
  for (auto& kv : precondGraphs_) cudaGraphExecDestroy(kv.second);
  if (hostScalars_) cudaFreeHost(hostScalars_);
  if (hostActive_) cudaFreeHost(hostActive_);
  if (hostBoxSums_) cudaFreeHost(hostBoxSums_);
}

int64_t Solver::numFaces(int l, int dir) const {
  int64_t n = 0;
  for (const Box& b : amr_[l].grids.boxes) n += userRegion(b, dir).numPts();
  return n;
}

const void* Solver::regionPlan(const LevelPlan& p, int faceDir, int* nreg, int64_t* total) {
  auto key = std::make_pair((const void*)&p, faceDir);
  auto it = regionCache_.find(key);
  if (it == regionCache_.end()) {
    std::vector<RegionCopy> rc;
    int64_t off = 0;
    for (size_t b = 0; b < p.grids.size(); ++b) {
      Box r = userRegion(p.grids[b], faceDir);
      RegionCopy c;
      c.box = (int)b;
      for (int k = 0; k < 3; ++k) {
        c.lo[k] = r.lo[k];
        c.hi[k] = r.hi[k];
      }
      c.srcOff = off;
      off += r.numPts();
      rc.push_back(c);
    }
    RegionPlan rp;
    rp.n = (int)rc.size();
    rp.total = off;
    rp.dev = upload(bufs_, rc, own_);
    ownSync();
    it = regionCache_.emplace(key, rp).first;
  }
  *nreg = it->second.n;
  *total = it->second.total;
  return it->second.dev;
}

double* Solver::staging(int64_t n) {
  if (!stage_ || stage_->bytes < (size_t)n * sizeof(double)) {
    if (s_ != own_) ck(cudaStreamSynchronize(s_), "staging");
    stage_.reset(new DevBuf(n * sizeof(double), own_));
    ownSync();
  }
  return (double*)stage_->p;
}

void Solver::scatterValid(const LevelPlan& p, const LevelDev& d, double* dev, const double* src, bool onDevice,
                          int faceDir) {
  int nreg;
  int64_t total;
  const RegionCopy* rc = (const RegionCopy*)regionPlan(p, faceDir, &nreg, &total);
  if (nreg == 0) return;
  const double* dsrc = src;
  if (!onDevice) {
    double* st = staging(total);
    ck(cudaMemcpyAsync(st, src, total * sizeof(double), cudaMemcpyHostToDevice, s_), "scatter h2d");
    dsrc = st;
  }
  k_scatter<<<nreg, 256, 0, s_>>>(d.boxes, rc, dev, dsrc, 1);
  ck(cudaGetLastError(), "scatter");
  ck(cudaStreamSynchronize(s_), "scatter sync");
}

void Solver::gatherValid(const LevelPlan& p, const LevelDev& d, const double* dev, double* dst, bool onDevice) {
  int nreg;
  int64_t total;
  const RegionCopy* rc = (const RegionCopy*)regionPlan(p, -1, &nreg, &total);
  if (nreg == 0) return;
  double* ddst = onDevice ? dst : staging(total);
  k_scatter<<<nreg, 256, 0, s_>>>(d.boxes, rc, const_cast<double*>(dev), ddst, 0);
  ck(cudaGetLastError(), "gather");
  if (!onDevice) ck(cudaMemcpyAsync(dst, ddst, total * sizeof(double), cudaMemcpyDeviceToHost, s_), "gather d2h");
  ck(cudaStreamSynchronize(s_), "gather sync");
}

void Solver::setRHS(int l, const double* src, bool onDevice) { scatterValid(amr_[l], amrDev_[l], lev_[l].rhs, src, onDevice, -1); }
void Solver::setPhi(int l, const double* src, bool onDevice) { scatterValid(amr_[l], amrDev_[l], lev_[l].phi, src, onDevice, -1); }
void Solver::getPhi(int l, double* dst, bool onDevice) { gatherValid(amr_[l], amrDev_[l], lev_[l].phi, dst, onDevice); }
void Solver::getRHS(int l, double* dst, bool onDevice) { gatherValid(amr_[l], amrDev_[l], lev_[l].rhs, dst, onDevice); }

void Solver::setACoef(int l, const double* src, bool onDevice) {
  if (!desc_.vc) throw std::runtime_error("cmg: a coefficient on a constant-coefficient operator");
  int64_t n = numValidCells(l);
  hostA_[l].resize(n);
  if (onDevice)
    ck(cudaMemcpy(hostA_[l].data(), src, n * sizeof(double), cudaMemcpyDeviceToHost), "a d2h");
  else
    std::memcpy(hostA_[l].data(), src, n * sizeof(double));
  scatterValid(amr_[l], amrDev_[l], lev_[l].a, hostA_[l].data(), false, -1);
}

void Solver::setBCoef(int l, int dir, const double* src, bool onDevice) {
  if (!desc_.vc) throw std::runtime_error("cmg: b coefficient on a constant-coefficient operator");
  int64_t n = numFaces(l, dir);
  hostB_[dir][l].resize(n);
  if (onDevice)
    ck(cudaMemcpy(hostB_[dir][l].data(), src, n * sizeof(double), cudaMemcpyDeviceToHost), "b d2h");
  else
    std::memcpy(hostB_[dir][l].data(), src, n * sizeof(double));
  scatterValid(amr_[l], amrDev_[l], lev_[l].b[dir], hostB_[dir][l].data(), false, dir);
}

}  // namespace cmg

namespace cmg {

namespace {

// Offsets of each box's block in the user-order arrays.
std::vector<int64_t> userOffsets(const Layout& g, int faceDir) {
  std::vector<int64_t> off(g.size() + 1, 0);
  for (size_t b = 0; b < g.size(); ++b) off[b + 1] = off[b] + userRegion(g[b], faceDir).numPts();
  return off;
}
inline int64_t userIdx(const Box& r, int i, int j, int k) {
  return (int64_t)(i - r.lo[0]) + (int64_t)r.size(0) * ((int64_t)(j - r.lo[1]) + (int64_t)r.size(1) * (k - r.lo[2]));
}

// lambda = 1 / (alpha a + sum_d scale beta (b_hi + b_lo)), VCAMRPoissonOp2::resetLambda
// (AMRElliptic/VCAMRPoissonOp2.cpp:283-318) with SUMFACES (VCAMRPoissonOpF.ChF:498-525).
std::vector<double> computeLambda(const Layout& g, const std::vector<double>& a, const std::vector<double>* b,
                                  double alpha, double beta, double dx) {
  std::vector<double> lam(a.size());
  auto ao = userOffsets(g, -1);
  std::vector<int64_t> bo[3];
  for (int d = 0; d < 3; ++d) bo[d] = userOffsets(g, d);
  const double scale = 1.0 / (dx * dx);
  for (size_t bx = 0; bx < g.size(); ++bx) {
    const Box& B = g[bx];
    for (int k = B.lo[2]; k <= B.hi[2]; ++k)
      for (int j = B.lo[1]; j <= B.hi[1]; ++j)
        for (int i = B.lo[0]; i <= B.hi[0]; ++i) {
          int64_t c = ao[bx] + userIdx(B, i, j, k);
          double l = a[c] * alpha;
          for (int d = 0; d < 3; ++d) {
            Box fr = userRegion(B, d);
            int hi[3] = {i, j, k};
            hi[d] += 1;
            double sumVal = b[d][bo[d][bx] + userIdx(fr, hi[0], hi[1], hi[2])] + b[d][bo[d][bx] + userIdx(fr, i, j, k)];
            l = l + scale * beta * sumVal;
          }
          lam[c] = 1.0 / l;
        }
  }
  return lam;
}

// CoarseAverage (AverageF.ChF:9-163) of cell data by ratio r, box b -> box b.
std::vector<double> averageCells(const Layout& fine, const Layout& coarse, const std::vector<double>& f, int r) {
  auto fo = userOffsets(fine, -1), co = userOffsets(coarse, -1);
  std::vector<double> out(co.back());
  const double refScale = 1.0 / (double)(r * r * r);
  for (size_t bx = 0; bx < coarse.size(); ++bx) {
    const Box& C = coarse[bx];
    const Box& F = fine[bx];
    for (int k = C.lo[2]; k <= C.hi[2]; ++k)
      for (int j = C.lo[1]; j <= C.hi[1]; ++j)
        for (int i = C.lo[0]; i <= C.hi[0]; ++i) {
          double s = 0.0;
          bool first = true;
          for (int c = 0; c < r; ++c)
            for (int b = 0; b < r; ++b)
              for (int a = 0; a < r; ++a) {
                double v = f[fo[bx] + userIdx(F, i * r + a, j * r + b, k * r + c)];
                s = first ? v : s + v;
                first = false;
              }
          out[co[bx] + userIdx(C, i, j, k)] = (r == 2 || r == 4) ? refScale * s : s * refScale;
        }
  }
  return out;
}

// CoarseAverageFace arithmetic (AverageFaceF.ChF:22-66) by ratio r.
std::vector<double> averageFaces(const Layout& fine, const Layout& coarse, const std::vector<double>& f, int r, int dir) {
  auto fo = userOffsets(fine, dir), co = userOffsets(coarse, dir);
  std::vector<double> out(co.back());
  const double base = 1.0 / (double)r;
  const double refScale = base * base;
  int ext[3] = {r, r, r};
  ext[dir] = 1;
  for (size_t bx = 0; bx < coarse.size(); ++bx) {
    Box C = userRegion(coarse[bx], dir);
    Box F = userRegion(fine[bx], dir);
    for (int k = C.lo[2]; k <= C.hi[2]; ++k)
      for (int j = C.lo[1]; j <= C.hi[1]; ++j)
        for (int i = C.lo[0]; i <= C.hi[0]; ++i) {
          double s = 0;
          for (int c = 0; c < ext[2]; ++c)
            for (int b = 0; b < ext[1]; ++b)
              for (int a = 0; a < ext[0]; ++a) s = s + f[fo[bx] + userIdx(F, i * r + a, j * r + b, k * r + c)];
          out[co[bx] + userIdx(C, i, j, k)] = refScale * s;
        }
  }
  return out;
}

}  // namespace

void Solver::finalizeCoefficients() {
  if (!desc_.vc) return;
  for (int l = 0; l < numLevels(); ++l) {
    if (hostA_[l].empty() || hostB_[0][l].empty() || hostB_[1][l].empty() || hostB_[2][l].empty())
      throw std::runtime_error("cmg: coefficients missing on a level");
    std::vector<double> b[3] = {hostB_[0][l], hostB_[1][l], hostB_[2][l]};
    auto lam = computeLambda(amr_[l].grids, hostA_[l], b, desc_.alpha, desc_.beta, amr_[l].dx);
    scatterValid(amr_[l], amrDev_[l], lev_[l].lambda, lam.data(), false, -1);
  }
  // Multigrid depths average the level-0 coefficients directly by 2^depth
  // (VCAMRPoissonOp2Factory::MGnewOp, AMRElliptic/VCAMRPoissonOp2.cpp:1019-1058).
  for (size_t d = 0; d < mg_.size(); ++d) {
    int r = 2 << d;
    auto a = averageCells(amr_[0].grids, mg_[d].grids, hostA_[0], r);
    std::vector<double> b[3];
    for (int k = 0; k < 3; ++k) b[k] = averageFaces(amr_[0].grids, mg_[d].grids, hostB_[k][0], r, k);
    scatterValid(mg_[d], mgDev_[d], mgf_[d].a, a.data(), false, -1);
    for (int k = 0; k < 3; ++k) scatterValid(mg_[d], mgDev_[d], mgf_[d].b[k], b[k].data(), false, k);
    auto lam = computeLambda(mg_[d].grids, a, b, desc_.alpha, desc_.beta, mg_[d].dx);
    scatterValid(mg_[d], mgDev_[d], mgf_[d].lambda, lam.data(), false, -1);
  }
  coef32Stale_ = true;
  // Compact copies of the bottom level's coefficients for the bottom solve.
  Coef<double> cb = coefMG((int)mg_.size());
  for (BottomWork& w : bottoms_) {
    gatherSlots(w, cb.a, w.a, s_);
    for (int k = 0; k < 3; ++k) gatherSlots(w, cb.b[k], w.b[k], s_);
    gatherSlots(w, cb.lambda, w.lam, s_);
  }
  ck(cudaStreamSynchronize(s_), "bottom coefficients");
}

void Solver::fillSyntheticDevice(uint64_t seed) {
  for (int l = 0; l < numLevels(); ++l)
    fillSyntheticLevel(amrDev_[l], seed, lev_[l].rhs, desc_.vc ? lev_[l].a : nullptr, desc_.vc ? lev_[l].b : nullptr,
                       s_);
  if (desc_.vc) {
    for (int l = 0; l < numLevels(); ++l)
      lambdaLevel(amrDev_[l], lev_[l].a, lev_[l].b, desc_.alpha, desc_.beta, lev_[l].lambda, s_);
    for (size_t d = 0; d < mg_.size(); ++d) {
      averageCoefficients(amrDev_[0], mgDev_[d], 2 << d, lev_[0].a, lev_[0].b, mgf_[d].a, mgf_[d].b, s_);
      lambdaLevel(mgDev_[d], mgf_[d].a, mgf_[d].b, desc_.alpha, desc_.beta, mgf_[d].lambda, s_);
    }
    coef32Stale_ = true;
    Coef<double> cb = coefMG((int)mg_.size());
    for (BottomWork& w : bottoms_) {
      gatherSlots(w, cb.a, w.a, s_);
      for (int k = 0; k < 3; ++k) gatherSlots(w, cb.b[k], w.b[k], s_);
      gatherSlots(w, cb.lambda, w.lam, s_);
    }
  }
  ck(cudaStreamSynchronize(s_), "device inputs");
}

void Solver::fillSyntheticForest(const std::vector<uint64_t>& seeds) {
  if ((int)seeds.size() != nh_) throw std::invalid_argument("cmg: one seed per hierarchy");
  for (int l = 0; l < numLevels(); ++l) {
    const LevelPlan& p = amr_[l];
    for (int k = 0; k < nh_; ++k) {
      // boxes and chunks of hierarchy k (both ordered by hierarchy)
      int b0 = 0, b1 = 0, c0 = 0, c1 = 0;
      if (nh_ == 1) {
        b1 = (int)p.boxes.size();
        c1 = (int)p.chunksAll.size();
      } else {
        b0 = (int)(std::lower_bound(p.boxHier.begin(), p.boxHier.end(), k) - p.boxHier.begin());
        b1 = (int)(std::upper_bound(p.boxHier.begin(), p.boxHier.end(), k) - p.boxHier.begin());
        auto byBox = [](const Chunk& c, int b) { return c.box < b; };
        c0 = (int)(std::lower_bound(p.chunksAll.begin(), p.chunksAll.end(), b0, byBox) - p.chunksAll.begin());
        c1 = (int)(std::lower_bound(p.chunksAll.begin(), p.chunksAll.end(), b1, byBox) - p.chunksAll.begin());
      }
      fillSyntheticBoxes(amrDev_[l], seeds[k], lev_[l].rhs, desc_.vc ? lev_[l].a : nullptr,
                         desc_.vc ? lev_[l].b : nullptr, b0, b1, c0, c1, s_);
    }
  }
  if (desc_.vc) {
    for (int l = 0; l < numLevels(); ++l)
      lambdaLevel(amrDev_[l], lev_[l].a, lev_[l].b, desc_.alpha, desc_.beta, lev_[l].lambda, s_);
    for (size_t d = 0; d < mg_.size(); ++d) {
      averageCoefficients(amrDev_[0], mgDev_[d], 2 << d, lev_[0].a, lev_[0].b, mgf_[d].a, mgf_[d].b, s_);
      lambdaLevel(mgDev_[d], mgf_[d].a, mgf_[d].b, desc_.alpha, desc_.beta, mgf_[d].lambda, s_);
    }
    coef32Stale_ = true;
    Coef<double> cb = coefMG((int)mg_.size());
    for (BottomWork& w : bottoms_) {
      gatherSlots(w, cb.a, w.a, s_);
      for (int k = 0; k < 3; ++k) gatherSlots(w, cb.b[k], w.b[k], s_);
      gatherSlots(w, cb.lambda, w.lam, s_);
    }
  }
  ck(cudaStreamSynchronize(s_), "device inputs");
}

int64_t Solver::hierarchyCells(int k, int l) const {
  if (k < 0 || k >= nh_ || l < 0 || l >= numLevels()) throw std::invalid_argument("cmg: hierarchy or level out of range");
  const LevelPlan& p = amr_[l];
  if (nh_ == 1) return p.grids.numCells();
  int64_t n = 0;
  for (size_t b = 0; b < p.boxes.size(); ++b)
    if (p.boxHier[b] == k) n += p.grids.boxes[b].numPts();
  return n;
}

Coef<double> Solver::coefAMR(int l) const {
  Coef<double> c;
  c.vc = desc_.vc;
  c.alpha = desc_.alpha;
  c.beta = desc_.beta;
  c.a = lev_[l].a;
  for (int d = 0; d < 3; ++d) c.b[d] = lev_[l].b[d];
  c.lambda = lev_[l].lambda;
  return c;
}

Coef<double> Solver::coefMG(int d) const {
  if (d == 0) return coefAMR(0);
  Coef<double> c;
  c.vc = desc_.vc;
  c.alpha = desc_.alpha;
  c.beta = desc_.beta;
  const LevelFields& f = mgf_[d - 1];
  c.a = f.a;
  for (int k = 0; k < 3; ++k) c.b[k] = f.b[k];
  c.lambda = f.lambda;
  return c;
}

}  // namespace cmg

namespace cmg {

template <>
std::vector<Solver::FieldsT<double>>& Solver::levF<double>() { return lev_; }
template <>
std::vector<Solver::FieldsT<float>>& Solver::levF<float>() { return lev32_; }
template <>
std::vector<Solver::FieldsT<double>>& Solver::mgF<double>() { return mgf_; }
template <>
std::vector<Solver::FieldsT<float>>& Solver::mgF<float>() { return mgf32_; }

template <class T>
Coef<T> Solver::coefA(int l) {
  Coef<T> c;
  c.vc = desc_.vc;
  c.alpha = desc_.alpha;
  c.beta = desc_.beta;
  const FieldsT<T>& f = levF<T>()[l];
  c.a = f.a;
  for (int d = 0; d < 3; ++d) c.b[d] = f.b[d];
  c.lambda = f.lambda;
  return c;
}

template <class T>
Coef<T> Solver::coefM(int d) {
  if (d == 0) return coefA<T>(0);
  Coef<T> c;
  c.vc = desc_.vc;
  c.alpha = desc_.alpha;
  c.beta = desc_.beta;
  const FieldsT<T>& f = mgF<T>()[d - 1];
  c.a = f.a;
  for (int k = 0; k < 3; ++k) c.b[k] = f.b[k];
  c.lambda = f.lambda;
  return c;
}

template <class T>
void Solver::zeroField(const LevelDev& L, T* f) {
  ck(cudaMemsetAsync(f, 0, L.nelem * sizeof(T), s_), "zero");
}
template <class T>
void Solver::copyField(const LevelDev& L, T* dst, const T* src) {
  ck(cudaMemcpyAsync(dst, src, L.nelem * sizeof(T), cudaMemcpyDeviceToDevice, s_), "copy");
}

// AMRPoissonOp::levelGSRB / VCAMRPoissonOp2::levelGSRB: per colour,
// homogeneous CF interpolation + exchange + BC, then the colour update.
// Algorithmic bytes of one colour pass over the red-black ordered layout,
// per cell of the level: half a word each for the updated colour's phi read,
// phi write and rhs, and the other colour's phi read (constant
// coefficients, 2 words); variable coefficients add half a word each for
// a and lambda and a full word for each of the three face arrays, since
// every face borders one cell of each colour (6 words).
template <class T>
void Solver::relaxLevel(const LevelDev& L, double cells, const Coef<T>& c, T* phi, const T* rhs, int n, int cls,
                        int variant) {
  const double bytes = cells * sizeof(T) * (c.vc ? 6.0 : 2.0);
  if (variant == 2) {
    timed(cls, bytes * 2 * n, [&]() { relaxBlock(L, phi, rhs, c, n, s_); });
    return;
  }
  if (variant == 3) {
    // Fused sweep: phi read and written once, rhs, a, lambda and the three
    // face arrays read once per sweep (8 words VC, 3 constant coefficients).
    const double sweepBytes = cells * sizeof(T) * (c.vc ? 8.0 : 3.0);
    for (int it = 0; it < n; ++it) timed(cls, sweepBytes, [&]() { gsrbSweepFused(L, phi, rhs, c, s_); });
    return;
  }
  // without per-chunk lists (large levels) the prefill variant is the fill one
  const bool inl = variant == 1 && (L.chGhost[0] != nullptr || L.nColor[0] == 0);
  for (int it = 0; it < n; ++it)
    for (int color = 0; color <= 1; ++color) {
      if (!inl) fill(L, phi, true, 1 - color);
      timed(cls, bytes, [&]() { gsrb(L, phi, rhs, c, color, s_, inl); });
    }
}

template <class T>
void Solver::relaxAMR(int l, T* phi, const T* rhs, int n) {
  const int finest = (int)amr_.size() - 1;
  relaxLevel(amrDev_[l], (double)amr_[l].grids.numCells(), coefA<T>(l), phi, rhs, n,
             l == finest ? P_RELAX_FINE : P_RELAX, inlineA_[l]);
}

template <class T>
void Solver::relaxMG(int d, T* phi, const T* rhs, int n) {
  if (d == 0) return relaxAMR(0, phi, rhs, n);
  relaxLevel(mgDev_[d - 1], (double)mg_[d - 1].grids.numCells(), coefM<T>(d), phi, rhs, n, P_RELAX,
             inlineM_[d - 1]);
}

// Relaxation autotuner: per AMR level and multigrid depth, time one red-black
// sweep with a ghost fill before each colour pass and one with the face
// ghosts evaluated inside the pass (identical results), on the level's
// scratch fields, and keep the faster.  Runs once per hierarchy, before its
// first solve, unless a mode is forced.
// The fill variant (0) unless another is faster by more than 2%: timings
// within that margin are noise, and the plain pass keeps one choice from
// run to run.
static int pickVariant(const float* t, int n) {
  int best = 0;
  for (int v = 1; v < n; ++v)
    if (t[v] < 0.98f * t[best]) best = v;
  return best;
}

void Solver::tuneRelaxation() {
  tuned_ = true;
  tuneMs_.clear();
  const char forced = relaxMode_ == 2 ? 1 : relaxMode_ == 3 ? 3 : 0;
  if (forced == 3) ensureDeferred();
  if (relaxMode_ == 0 || relaxMode_ == 2) ensureChunkGhosts();
  // The variants the tuner compares on a level: the prefill one where the
  // level has its per-chunk lists, the one-block one on small levels; the
  // fused sweep (slower on every level measured) only when forced.
  auto offered = [&](const LevelDev& L, double cells, int v) {
    if (v == 1) return L.chGhost[0] != nullptr;
    if (v == 2) return cells <= kBlockRelaxMaxCells;
    return v != 3;
  };
  inlineA_.assign(amr_.size(), forced);
  inlineM_.assign(mg_.size(), forced);
  if (relaxMode_ != 0) return;
  cudaEvent_t e[3];
  for (auto& x : e) ck(cudaEventCreate(&x), "event");
  const bool prof = profOn_;
  profOn_ = false;
  auto timeOne = [&](const LevelDev& L, double cells, const Coef<double>& c, double* phi, const double* rhs,
                     int variant) {
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      ck(cudaEventRecord(e[0], s_), "event");
      relaxLevel(L, cells, c, phi, rhs, 4, P_RELAX, variant);
      ck(cudaEventRecord(e[1], s_), "event");
      ck(cudaEventSynchronize(e[1]), "event sync");
      float ms = 0;
      ck(cudaEventElapsedTime(&ms, e[0], e[1]), "event time");
      best = std::min(best, ms);
    }
    return best;
  };
  for (size_t l = 0; l < amr_.size(); ++l) {
    const double cells = (double)amr_[l].grids.numCells();
    Coef<double> c = coefAMR((int)l);
    float t[kRelaxVariants];
    for (int v = 0; v < kRelaxVariants; ++v)
      t[v] = offered(amrDev_[l], cells, v) ? timeOne(amrDev_[l], cells, c, lev_[l].corr, lev_[l].res, v) : 1e30f;
    inlineA_[l] = (char)pickVariant(t, kRelaxVariants);
    tuneMs_.push_back({t[0], *std::min_element(t + 1, t + kRelaxVariants)});
    zeroField(amrDev_[l], lev_[l].corr);
  }
  for (size_t d = 0; d < mg_.size(); ++d) {
    const double cells = (double)mg_[d].grids.numCells();
    Coef<double> c = coefMG((int)d + 1);
    float t[kRelaxVariants];
    for (int v = 0; v < kRelaxVariants; ++v)
      t[v] = offered(mgDev_[d], cells, v) ? timeOne(mgDev_[d], cells, c, mgf_[d].corr, mgf_[d].res, v) : 1e30f;
    inlineM_[d] = (char)pickVariant(t, kRelaxVariants);
    tuneMs_.push_back({t[0], *std::min_element(t + 1, t + kRelaxVariants)});
    zeroField(mgDev_[d], mgf_[d].corr);
  }
  profOn_ = prof;
  for (auto& x : e) cudaEventDestroy(x);
}

void Solver::relaxVariants(std::vector<int>& inl, std::vector<float>& msFill, std::vector<float>& msInline) {
  if (!tuned_) tuneRelaxation();
  inl.clear();
  msFill.clear();
  msInline.clear();
  for (char c : inlineA_) inl.push_back(c);
  for (char c : inlineM_) inl.push_back(c);  // 0 fills, 1 in-pass ghosts, 2 one-block sweeps
  for (auto& t : tuneMs_) {
    msFill.push_back(t.first);
    msInline.push_back(t.second);
  }
}

void Solver::setAlphaAndBeta(double alpha, double beta) {
  if (desc_.vc) {
    desc_.alpha = alpha;
    desc_.beta = beta;
    for (int l = 0; l < numLevels(); ++l)
      lambdaLevel(amrDev_[l], lev_[l].a, lev_[l].b, desc_.alpha, desc_.beta, lev_[l].lambda, s_);
    for (size_t d = 0; d < mg_.size(); ++d)
      lambdaLevel(mgDev_[d], mgf_[d].a, mgf_[d].b, desc_.alpha, desc_.beta, mgf_[d].lambda, s_);
    for (BottomWork& w : bottoms_) gatherSlots(w, coefMG((int)mg_.size()).lambda, w.lam, s_);
    coef32Stale_ = true;
  } else {
    desc_.alpha = alpha * alpha0_;
    desc_.beta = beta * beta0_;
  }
  ck(cudaStreamSynchronize(s_), "alpha and beta");
}

std::vector<SolveResult> Solver::backwardEuler(const SolveParams& p, double dt, int nsteps, bool zeroPhi) {
  needSingle();
  if (nsteps < 0) throw std::invalid_argument("cmg: negative step count");
  const int nlev = numLevels();
  if (src_.empty()) {
    src_.resize(nlev);
    for (int l = 0; l < nlev; ++l) src_[l] = alloc(amr_[l].nelem);
  }
  for (int l = 0; l < nlev; ++l) copyField(amrDev_[l], src_[l], lev_[l].rhs);
  std::vector<SolveResult> out;
  for (int n = 0; n < nsteps; ++n) {
    // createEulerRHS, then phiNew = phiOld (in place), solveHelm.
    for (int l = 0; l < nlev; ++l)
      eulerRHS(lev_[l].rhs, lev_[l].phi, desc_.vc ? lev_[l].a : nullptr, src_[l], dt, amr_[l].nelem, s_);
    setAlphaAndBeta(1.0, -dt);
    out.push_back(solve(p, zeroPhi));
  }
  for (int l = 0; l < nlev; ++l) copyField(amrDev_[l], lev_[l].rhs, src_[l]);
  ck(cudaStreamSynchronize(s_), "backward Euler");
  return out;
}

std::vector<SolveResult> Solver::tga(const SolveParams& p, double dt, int nsteps) {
  needSingle();
  if (nsteps < 0) throw std::invalid_argument("cmg: negative step count");
  const int nlev = numLevels();
  // AMRTGA::setMu (AMRTGA.H:351-366).
  const double tgaEpsilon = 1.e-12;
  const double a = 2.0 - std::sqrt(2.0) - tgaEpsilon;
  const double mu1 = (a - std::sqrt(a * a - 4.0 * a + 2.0)) / 2.0;
  const double mu2 = (a + std::sqrt(a * a - 4.0 * a + 2.0)) / 2.0;
  const double mu3 = (1.0 - a);
  const double mu4 = 0.5 - a;
  if (src_.empty()) {
    src_.resize(nlev);
    for (int l = 0; l < nlev; ++l) src_[l] = alloc(amr_[l].nelem);
  }
  for (int l = 0; l < nlev; ++l) copyField(amrDev_[l], src_[l], lev_[l].rhs);
  MLVec phiOld = mlVec(0), srct = mlVec(1), rhst = mlVec(2);
  MLVec phiNew(nlev), src(nlev);
  for (int l = 0; l < nlev; ++l) {
    phiNew[l] = lev_[l].phi;
    src[l] = src_[l];
  }
  auto aCoef = [&](int l) -> const double* { return desc_.vc ? lev_[l].a : nullptr; };
  std::vector<SolveResult> out;
  for (int n = 0; n < nsteps; ++n) {
    mlAssign(phiOld, phiNew);
    for (int l = 0; l < nlev; ++l) tgaSource(srct[l], src[l], aCoef(l), amr_[l].nelem, s_);
    // applyHelm(rhst, srct, mu4): (a I + mu4 dt L) S/a, then times dt.
    setAlphaAndBeta(1.0, mu4 * dt);
    mlApplyOp(rhst, srct);
    mlScale(rhst, dt);
    // applyHelm(phiNew, phiOld, mu3), added to rhst.
    setAlphaAndBeta(1.0, mu3 * dt);
    mlApplyOp(phiNew, phiOld);
    mlIncr(rhst, phiNew, 1.0);
    // solveHelm(phiNew, rhst, mu2) from phiOld.
    mlAssign(phiNew, phiOld);
    setAlphaAndBeta(1.0, -mu2 * dt);
    for (int l = 0; l < nlev; ++l) copyField(amrDev_[l], lev_[l].rhs, rhst[l]);
    out.push_back(solve(p, false));
    // rhst = diagonalScale(phiNew); solveHelm(phiNew, rhst, mu1) from phiOld.
    mlAssign(rhst, phiNew);
    if (desc_.vc)
      for (int l = 0; l < nlev; ++l) multField(rhst[l], lev_[l].a, amr_[l].nelem, s_);
    mlAssign(phiNew, phiOld);
    setAlphaAndBeta(1.0, -mu1 * dt);
    for (int l = 0; l < nlev; ++l) copyField(amrDev_[l], lev_[l].rhs, rhst[l]);
    out.push_back(solve(p, false));
  }
  for (int l = 0; l < nlev; ++l) copyField(amrDev_[l], lev_[l].rhs, src_[l]);
  ck(cudaStreamSynchronize(s_), "TGA");
  return out;
}

void Solver::setBottomConfig(const BottomConfig& c) {
  if (c.kind != 0 && c.kind != 1) throw std::invalid_argument("cmg: bottom solver is BiCGStab (0) or relaxation (1)");
  if (c.normType != 0 && c.normType != 2) throw std::invalid_argument("cmg: bottom solver norm type is 0 or 2");
  if (c.imax < 0 || c.numRestarts < 0) throw std::invalid_argument("cmg: negative bottom solver iteration limit");
  bottomCfg_ = c;
  // captured bottom launches hold the old parameters
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
  graphs_.clear();
  for (auto& kv : precondGraphs_) cudaGraphExecDestroy(kv.second);
  precondGraphs_.clear();
}

void Solver::setBottomGrid(int mode) {
  if (mode < -1 || mode > 1) throw std::invalid_argument("cmg: bottom grid mode is -1 (automatic), 0 or 1");
  // One hierarchy with a large bottom level: the solve spreads over the
  // device in one cooperative launch (below that, one block is faster).
  int blocks = 0;
  if (nh_ == 1 && mode != 0 && (mode == 1 || bottoms_[0].nv >= kBottomGridMinCells)) {
    BottomWork& w = bottoms_[0];
    blocks = bottomGridBlocks(w.nv);
    if (!w.gscal) {
      const int nPart = std::max(w.nbox, blocks * bottomGridThreads() / 32);
      w.gpart = alloc(nPart);
      w.gpart2 = alloc(nPart);
      w.gscal = alloc(8);
      dBottoms_ = upload(bufs_, bottoms_, s_);
    }
  }
  if (blocks == bottomGrid_) return;
  bottomGrid_ = blocks;
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
  graphs_.clear();
  for (auto& kv : precondGraphs_) cudaGraphExecDestroy(kv.second);
  precondGraphs_.clear();
}

void Solver::ensureChunkGhosts() {
  auto one = [&](LevelPlan& p, LevelDev& d) {
    const bool hadRules = !p.faceOff.empty();
    if (!cmg::ensureChunkGhosts(p)) return;
    if (!hadRules) {
      d.faceRules = upload(bufs_, p.faceRules, s_);
      d.faceOff = upload(bufs_, p.faceOff, s_);
    }
    for (int c = 0; c < 2; ++c) {
      d.chGhost[c] = upload(bufs_, p.chunkGhost[c], s_);
      d.chGhostStart[c] = upload(bufs_, p.chunkGhostStart[c], s_);
    }
  };
  for (size_t l = 0; l < amr_.size(); ++l) one(amr_[l], amrDev_[l]);
  for (size_t d = 0; d < mg_.size(); ++d) one(mg_[d], mgDev_[d]);
  ck(cudaStreamSynchronize(s_), "chunk ghost lists");
}

void Solver::ensureDeferred() {
  auto one = [&](LevelPlan& p, LevelDev& d) {
    if (d.deferred || p.grids.size() == 0) return;
    if (ensureFaceRules(p)) {
      d.faceRules = upload(bufs_, p.faceRules, s_);
      d.faceOff = upload(bufs_, p.faceOff, s_);
    }
    buildDeferred(p);
    d.deferred = upload(bufs_, p.deferred, s_);
    d.nDeferred = (int)p.deferred.size();
  };
  for (size_t l = 0; l < amr_.size(); ++l) one(amr_[l], amrDev_[l]);
  for (size_t d = 0; d < mg_.size(); ++d) one(mg_[d], mgDev_[d]);
  ck(cudaStreamSynchronize(s_), "deferred lists");
}

void Solver::setRelaxMode(int mode) {
  if (mode < 0 || mode > 3)
    throw std::invalid_argument("cmg: relaxation mode is 0 (tuned), 1 (fills), 2 (inline) or 3 (fused sweeps)");
  relaxMode_ = mode;
  tuned_ = false;
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
  graphs_.clear();
  for (auto& kv : precondGraphs_) cudaGraphExecDestroy(kv.second);
  precondGraphs_.clear();
}

// Ghost fill, timed as its own class: every ghost cell filled written once
// and its source read once (two words per cell; half the cells for a
// one-colour fill).
template <class T>
void Solver::fill(const LevelDev& L, T* f, bool withCF, int par) {
  const double bytes = (par >= 0 ? 1.0 : 2.0) * sizeof(T) * (withCF ? L.nCellsGhost : L.nCellsExchBC);
  timed(P_GHOST, bytes, [&]() { ghostFill(L, f, withCF, s_, par); });
}

// AMRMultiGrid::computeAMRResidualLevel (AMRMultiGrid.H:836-892).
template <class T>
void Solver::amrResidualLevel(int ilev, int lmax, T* const* res, T* const* phi, T* const* rhs) {
  const LevelDev& L = amrDev_[ilev];
  Coef<T> c = coefA<T>(ilev);
  const double w = sizeof(T);
  if (lmax == 0) {
    // residual(): homogeneous CF (none on level 0), then residualI.
    fill(L, phi[0], true);
    timed(P_OP, amr_[0].grids.numCells() * w * (desc_.vc ? 7.0 : 3.0), [&]() { residual(L, res[0], phi[0], rhs[0], c, s_); });
    return;
  }
  if (ilev == lmax) {
    // AMRResidualNF: coarse-fine interpolation, then residualI.
    quadCF(L, phi[ilev], phi[ilev - 1], s_);
    fill(L, phi[ilev], false);
    timed(P_OP, amr_[ilev].grids.numCells() * w * (desc_.vc ? 7.0 : 3.0), [&]() { residual(L, res[ilev], phi[ilev], rhs[ilev], c, s_); });
    return;
  }
  // AMRResidual(NC): [CF interpolation], applyOpI, reflux, axby(-1, 1).
  if (ilev > 0) quadCF(L, phi[ilev], phi[ilev - 1], s_);
  fill(L, phi[ilev], false);
  timed(P_OP, amr_[ilev].grids.numCells() * w * (desc_.vc ? 6.0 : 2.0), [&]() { applyOp(L, res[ilev], phi[ilev], c, s_); });
  quadCF(amrDev_[ilev + 1], phi[ilev + 1], phi[ilev], s_);
  reflux(L, res[ilev], phi[ilev], phi[ilev + 1], c, coefA<T>(ilev + 1), s_);
  negAdd(L, res[ilev], res[ilev], rhs[ilev], s_);
}

// AMRMultiGrid::computeAMRResidual (AMRMultiGrid.H:682-736).
double Solver::computeAMRResidual(std::vector<double*>& res, std::vector<double*>& phi, std::vector<double*>& rhs,
                                  int lmax) {
  launchAMRResidual(res, phi, rhs, lmax);
  return readNorm();
}

// The device work of computeAMRResidual: residuals, zeroCovered, max-norm
// into dNorm_ (no host synchronisation, so it can be captured).
void Solver::launchAMRResidual(std::vector<double*>& res, std::vector<double*>& phi, std::vector<double*>& rhs,
                               int lmax) {
  ck(cudaMemsetAsync(dNorm_, 0, nh_ * sizeof(double), s_), "norm reset");
  for (int ilev = 0; ilev <= lmax; ++ilev) {
    amrResidualLevel<double>(ilev, lmax, res.data(), phi.data(), rhs.data());
    if (ilev != lmax) zeroCovered(amrDev_[ilev], res[ilev], s_);
    maxNorm(amrDev_[ilev], res[ilev], dNorm_, s_);
  }
}

// Through pinned host memory, so that the copy is a plain stream operation
// and concurrent solves on other streams are not serialised behind it.
double Solver::readNorm() {
  ck(cudaMemcpyAsync(&hostScalars_[0], dNorm_, sizeof(double), cudaMemcpyDeviceToHost, s_), "norm d2h");
  ck(cudaStreamSynchronize(s_), "norm sync");
  return hostScalars_[0];
}

std::vector<double> Solver::readNorms() {
  double* h = hostScalars_ + 2;
  ck(cudaMemcpyAsync(h, dNorm_, nh_ * sizeof(double), cudaMemcpyDeviceToHost, s_), "norm d2h");
  ck(cudaStreamSynchronize(s_), "norm sync");
  return std::vector<double>(h, h + nh_);
}

// BiCGStab bottom solve in FP64 whatever the V-cycle's precision: an FP32
// V-cycle hands its correction and residual over through the FP64 fields of
// the bottom level (free during the FP32 cycle) and takes the result back.
template <>
void Solver::bottom<double>(int depth, double* corr, double* res) {
  const LevelDev& L = depth == 0 ? amrDev_[0] : mgDev_[depth - 1];
  timed(P_BOTTOM, 0.0, [&]() {
    bottomSolve(L, corr, res, coefMG(depth), dBottoms_, nh_, maxBottomBoxes_, bottomCfg_, sp_.eps, dMetric_, s_,
                dEps_, bottomGrid_);
  });
}
template <>
void Solver::bottom<float>(int depth, float* corr, float* res) {
  const LevelDev& L = depth == 0 ? amrDev_[0] : mgDev_[depth - 1];
  double* corr64 = depth == 0 ? lev_[0].corr : mgf_[depth - 1].corr;
  double* res64 = depth == 0 ? lev_[0].res : mgf_[depth - 1].res;
  convert(corr64, corr, L.nelem, s_);
  convert(res64, res, L.nelem, s_);
  timed(P_BOTTOM, 0.0, [&]() {
    bottomSolve(L, corr64, res64, coefMG(depth), dBottoms_, nh_, maxBottomBoxes_, bottomCfg_, sp_.eps, dMetric_,
                s_, dEps_, bottomGrid_);
  });
  convert(corr, corr64, L.nelem, s_);
}

// MultiGrid::cycle (MultiGrid.H:629-696), V-cycle (m_cycle = 1).
template <class T>
void Solver::mgCycle(int depth, T* corr, T* res) {
  const int D = 1 + (int)mg_.size();
  if (depth == D - 1) {
    if (bottomCells_ == 1) {
      relaxMG(depth, corr, res, 1);
    } else {
      relaxMG(depth, corr, res, sp_.bottom);
      bottom<T>(depth, corr, res);
    }
    return;
  }
  const LevelDev& F = depth == 0 ? amrDev_[0] : mgDev_[depth - 1];
  const LevelDev& C = mgDev_[depth];
  T* corrC = mgF<T>()[depth].corr;
  T* resC = mgF<T>()[depth].res;
  relaxMG(depth, corr, res, sp_.pre);
  // restrictResidual: homogeneous CF (none) + exchange + BC, RESTRICTRES.
  fill(F, corr, true);
  restrictMG(F, C, resC, corr, res, coefM<T>(depth), s_);
  zeroField(C, corrC);
  for (int img = 0; img < sp_.numMG; ++img) mgCycle(depth + 1, corrC, resC);
  prolongMG(F, C, corr, corrC, s_);
  relaxMG(depth, corr, res, sp_.post);
}

// AMRMultiGrid::AMRVCycle (AMRMultiGrid.H:1341-1419), l_base = 0.
template <class T>
void Solver::amrVCycle(int ilev, int lmax) {
  std::vector<FieldsT<T>>& lev = levF<T>();
  if (ilev == lmax)
    for (int l = 0; l <= lmax; ++l) {
      copyField(amrDev_[l], lev[l].res, lev[l].ures);
      zeroField(amrDev_[l], lev[l].corr);
    }
  if (lmax == 0) {
    mgCycle(0, lev[0].ucorr, lev[0].ures);
    return;
  }
  if (ilev == 0) {
    mgCycle(0, lev[0].corr, lev[0].res);
    incr(amrDev_[0], lev[0].ucorr, lev[0].corr, 1.0, s_);
    return;
  }
  const LevelDev& L = amrDev_[ilev];
  const LevelDev& Lc = amrDev_[ilev - 1];
  FieldsT<T>& f = lev[ilev];
  FieldsT<T>& fc = lev[ilev - 1];
  const double w = sizeof(T);
  relaxAMR(ilev, f.corr, f.res, sp_.pre);
  incr(L, f.ucorr, f.corr, 1.0, s_);
  zeroField(Lc, fc.corr);
  std::vector<T*> res(lmax + 1), ucorr(lmax + 1), ures(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    res[l] = lev[l].res;
    ucorr[l] = lev[l].ucorr;
    ures[l] = lev[l].ures;
  }
  amrResidualLevel<T>(ilev - 1, lmax, res.data(), ucorr.data(), ures.data());
  // AMRRestrictS: residual of the correction into the scratch (uberCorrection),
  // averaged straight onto the coarse residual (assignCopier).
  quadCF(L, f.corr, fc.corr, s_);
  fill(L, f.corr, false);
  timed(P_OP, amr_[ilev].grids.numCells() * w * (desc_.vc ? 7.0 : 3.0), [&]() { residual(L, f.ucorr, f.corr, f.res, coefA<T>(ilev), s_); });
  averageAMR(L, Lc, fc.res, f.ucorr, s_);
  for (int img = 0; img < sp_.numMG; ++img) amrVCycle<T>(ilev - 1, lmax);
  // AMRProlongS, AMRUpdateResidual, post-smoothing of the correction's correction.
  prolongAMR(L, Lc, f.corr, fc.corr, s_);
  quadCF(L, f.corr, fc.corr, s_);
  fill(L, f.corr, false);
  timed(P_OP, amr_[ilev].grids.numCells() * w * (desc_.vc ? 7.0 : 3.0), [&]() { residual(L, f.res, f.corr, f.res, coefA<T>(ilev), s_); });
  zeroField(L, f.ucorr);
  relaxAMR(ilev, f.ucorr, f.res, sp_.post);
  incrCopy(L, f.corr, f.ucorr, s_);  // corr += ucorr; ucorr = corr
}

template void Solver::amrVCycle<double>(int, int);
template void Solver::amrVCycle<float>(int, int);
// Used by the operator-level calls (levelops.cu) and the allocation-free
// residual norm (noalloc.cu).
template void Solver::amrResidualLevel<double>(int, int, double* const*, double* const*, double* const*);
template void Solver::relaxAMR<double>(int, double*, const double*, int);
template void Solver::relaxMG<double>(int, double*, const double*, int);

// ------------------------------------------------ BiCGStab over MultilevelLinearOp
// BiCGStabSolver<Vector<LevelData<FArrayBox>*>>::solve (BiCGStabSolver.H:199-515)
// over MultilevelLinearOp<FArrayBox> (MultilevelLinearOpI.H), the solve path of
// the variable-coefficient example.  Vectors are one device array per AMR
// level in the level's ghosted layout; the scalars (rho, alpha, beta, omega,
// norms) live on the host as in the reference, each dot product and norm read
// back once.

Solver::MLVec Solver::mlVec(int i) {
  if (mlVecs_.empty()) {
    const int nlev = numLevels();
    mlVecs_.assign(10, MLVec(nlev, nullptr));
    for (auto& v : mlVecs_)
      for (int l = 0; l < nlev; ++l) v[l] = alloc(amr_[l].nelem);
    size_t nb = 0;
    for (const LevelDev& L : amrDev_) nb += (size_t)L.nbox;
    dBoxSums_ = alloc(std::max<size_t>(nb, 1));
    ck(cudaMallocHost((void**)&hostBoxSums_, std::max<size_t>(nb, 1) * sizeof(double)), "pinned box sums");
  }
  return mlVecs_[i];
}

void Solver::mlZero(MLVec& x) {
  for (int l = 0; l < numLevels(); ++l) zeroField(amrDev_[l], x[l]);
}
void Solver::mlAssign(MLVec& dst, const MLVec& src) {
  for (int l = 0; l < numLevels(); ++l) copyField(amrDev_[l], dst[l], src[l]);
}
void Solver::mlIncr(MLVec& y, const MLVec& x, double scale) {
  for (int l = 0; l < numLevels(); ++l) incr(amrDev_[l], y[l], x[l], scale, s_);
}
void Solver::mlScale(MLVec& x, double scale) {
  for (int l = 0; l < numLevels(); ++l) scaleField(x[l], scale, amrDev_[l].nelem, s_);
}

// MultilevelLinearOp::residual: AMRResidual(NC/NF) or residual per level, in
// level order.  The homogeneous and inhomogeneous physical boundary
// conditions coincide for these zero-value Dirichlet faces.
void Solver::mlResidual(MLVec& lhs, MLVec& phi, MLVec& rhs) {
  const int lmax = numLevels() - 1;
  for (int l = 0; l <= lmax; ++l) amrResidualLevel<double>(l, lmax, lhs.data(), phi.data(), rhs.data());
}

// AMROperator / AMROperatorNC / AMROperatorNF / applyOp of one level
// (AMRPoissonOp.cpp:332-340, 790-858): coarse-fine interpolation from the
// coarser level, exchange and boundary values, the operator, and the
// flux-register correction from the finer level.
void Solver::amrOperatorLevel(int ilev, int lmax, MLVec& lhs, MLVec& phi) {
  const LevelDev& L = amrDev_[ilev];
  Coef<double> c = coefA<double>(ilev);
  if (ilev > 0) quadCF(L, phi[ilev], phi[ilev - 1], s_);
  fill(L, phi[ilev], false);
  timed(P_OP, amr_[ilev].grids.numCells() * 8.0 * (desc_.vc ? 6.0 : 2.0), [&]() { applyOp(L, lhs[ilev], phi[ilev], c, s_); });
  if (ilev < lmax) {
    quadCF(amrDev_[ilev + 1], phi[ilev + 1], phi[ilev], s_);
    reflux(L, lhs[ilev], phi[ilev], phi[ilev + 1], c, coefA<double>(ilev + 1), s_);
  }
}

void Solver::mlApplyOp(MLVec& lhs, MLVec& phi) {
  const int lmax = numLevels() - 1;
  for (int l = 0; l <= lmax; ++l) amrOperatorLevel(l, lmax, lhs, phi);
}

// MultilevelLinearOp::norm with order 0: the largest AMRNorm over the
// levels, each the max-norm of the level with the cells under the next finer
// level zeroed.
double Solver::mlNorm(const MLVec& x) {
  const int lmax = numLevels() - 1;
  MLVec tmp = mlVec(8);
  ck(cudaMemsetAsync(dNorm_, 0, sizeof(double), s_), "norm reset");
  for (int l = 0; l <= lmax; ++l) {
    const double* src = x[l];
    if (l < lmax) {
      copyField(amrDev_[l], tmp[l], x[l]);
      zeroCovered(amrDev_[l], tmp[l], s_);
      src = tmp[l];
    }
    maxNorm(amrDev_[l], src, dNorm_, s_);
  }
  return readNorm();
}

// MultilevelLinearOp::dotProduct: copies with the covered cells zeroed, per
// level LevelDataOps::dotProduct (box dot products summed in box order), each
// level scaled by dx^3 and summed coarse to fine.
double Solver::mlDot(const MLVec& x, const MLVec& y) {
  const int lmax = numLevels() - 1;
  MLVec ta = mlVec(8), tb = mlVec(9);
  int off = 0;
  for (int l = 0; l <= lmax; ++l) {
    const LevelDev& L = amrDev_[l];
    const double* a = x[l];
    const double* b = y[l];
    if (l < lmax) {
      copyField(L, ta[l], x[l]);
      zeroCovered(L, ta[l], s_);
      a = ta[l];
      if (y[l] == x[l]) {
        b = a;
      } else {
        copyField(L, tb[l], y[l]);
        zeroCovered(L, tb[l], s_);
        b = tb[l];
      }
    }
    boxDots(L, a, b, dBoxSums_ + off, s_);
    off += L.nbox;
  }
  ck(cudaMemcpyAsync(hostBoxSums_, dBoxSums_, std::max(off, 1) * sizeof(double), cudaMemcpyDeviceToHost, s_),
     "box sums d2h");
  ck(cudaStreamSynchronize(s_), "box sums sync");
  double prod = 0.0;
  off = 0;
  for (int l = 0; l <= lmax; ++l) {
    double val = 0.0;
    for (int b = 0; b < amrDev_[l].nbox; ++b) val += hostBoxSums_[off + b];
    off += amrDev_[l].nbox;
    const double dx = amr_[l].dx;
    const double scale = dx * dx * dx;
    val *= scale;
    prod += val;
  }
  return prod;
}

// MultilevelLinearOp::preCond with the multigrid preconditioner: mgIters
// times, the homogeneous residual of the current correction, one AMR
// V-cycle from a zero correction (AMRMultiGrid::AMRVCycle on the
// preconditioner's own scratch), and the increment.
void Solver::mlPreCondBody(MLVec& cor, MLVec& res, const MLSolveParams& p) {
  const int lmax = numLevels() - 1;
  MLVec ures(lmax + 1), ucorr(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    ures[l] = lev_[l].ures;
    ucorr[l] = lev_[l].ucorr;
  }
  for (int it = 0; it < p.mgIters; ++it) {
    mlResidual(ures, cor, res);
    mlZero(ucorr);
    amrVCycle<double>(lmax, lmax);
    mlIncr(cor, ucorr, 1.0);
  }
}

// The preconditioner call is one CUDA-graph replay when graphs are on (no
// host decision inside it; the bottom solve reads its metric from device
// memory).
void Solver::mlPreCond(MLVec& cor, MLVec& res, const MLSolveParams& p) {
  if (!useGraphs_ || profOn_) {
    mlPreCondBody(cor, res, p);
    return;
  }
  const auto key = std::make_tuple((const void*)cor[0], (const void*)res[0], p.mgIters, p.mgSmooth, desc_.alpha,
                                   desc_.beta);
  auto it = precondGraphs_.find(key);
  cudaGraphExec_t exec = nullptr;
  if (it != precondGraphs_.end()) {
    exec = it->second;
  } else {
    if (precondGraphs_.size() >= kMaxGraphs) {
      for (auto& kv : precondGraphs_) cudaGraphExecDestroy(kv.second);
      precondGraphs_.clear();
    }
    cudaGraph_t g = nullptr;
    const long long before = launchCount();
    ck(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      mlPreCondBody(cor, res, p);
    } catch (...) {
      cudaStreamEndCapture(s_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    ck(cudaStreamEndCapture(s_, &g), "end capture");
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    ck(e, "graph instantiate");
    precondGraphs_[key] = exec;
    graphLaunches_[exec] = launchCount() - before;
    addLaunches(-(launchCount() - before));
  }
  ck(cudaGraphLaunch(exec, s_), "graph launch");
  addLaunches(graphLaunches_[exec]);
}

void Solver::interpToFine(int l, bool pwc) {
  needSingle();
  if (l < 1 || l >= numLevels()) throw std::invalid_argument("cmg: fine interpolation needs a level in 1..finest");
  if (fineInterp_.size() < amr_.size()) fineInterp_.resize(amr_.size());
  if (!fineInterp_[l])
    fineInterp_[l].reset(
        new FineInterpOp(amr_[l - 1].grids.boxes, amr_[l - 1].index, amr_[l - 1].domain, amr_[l].grids.boxes, own_));
  fineInterp_[l]->setStream(s_);
  // algorithmic bytes: every fine cell written once, every coarse parent read once
  const double bytes = 9.0 * sizeof(double) / 8.0 * (double)fineInterp_[l]->fineCells();
  timed(P_FINEINTERP, bytes,
        [&]() { fineInterp_[l]->run(amrDev_[l - 1].boxes, lev_[l - 1].phi, amrDev_[l].boxes, lev_[l].phi, pwc); });
  ck(cudaStreamSynchronize(s_), "fine interpolation sync");
}

MLSolveResult Solver::solveMultilevelBiCGStab(const MLSolveParams& p, bool zeroPhi) {
  needSingle();
  if (p.mgIters < 0 || p.mgSmooth < 0 || p.imax < 0 || p.numRestarts < 0)
    throw std::invalid_argument("cmg: invalid BiCGStab parameters");
  if (!tuned_) tuneRelaxation();
  const int lmax = numLevels() - 1;
  // The preconditioner's AMRMultiGrid (MultilevelLinearOp::define): pre,
  // post and bottom smoothings m_num_mg_smooth, one V-cycle per call, and a
  // default BiCGStabSolver at the bottom (eps 1e-6, no convergence metric:
  // AMRVCycle is called directly, so setConvergenceMetrics never runs).
  const SolveParams saved = sp_;
  sp_ = SolveParams();
  sp_.pre = sp_.post = sp_.bottom = p.mgSmooth;
  sp_.numMG = 1;
  sp_.eps = 1e-6;
  hostScalars_[1] = -1.0;
  ck(cudaMemcpyAsync(dMetric_, &hostScalars_[1], sizeof(double), cudaMemcpyHostToDevice, s_), "metric");
  MLVec phi(lmax + 1), rhs(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    phi[l] = lev_[l].phi;
    rhs[l] = lev_[l].rhs;
  }
  if (zeroPhi) mlZero(phi);
  MLVec r = mlVec(0), rt = mlVec(1), e = mlVec(2), pv = mlVec(3), pt = mlVec(4), st = mlVec(5), t = mlVec(6),
        v = mlVec(7);
  MLSolveResult out;
  out.exitStatus = -1;
  int recount = 0;
  mlZero(r);
  mlResidual(r, phi, rhs);
  mlAssign(rt, r);
  mlZero(e);
  mlZero(pt);
  mlZero(st);
  int iter = 0;
  double rho[4] = {0, 0, 0, 0};
  double norm[2];
  norm[0] = mlNorm(r);
  const double initial_norm = norm[0];
  out.initialResidual = norm[0];
  out.finalResidual = norm[0];
  norm[1] = norm[0];
  double alpha[2] = {0, 0}, beta[2] = {0, 0}, omega[2] = {0, 0};
  bool init = true;
  int restarts = 0;
  while ((iter < p.imax && norm[0] > p.eps * norm[1]) && (norm[1] > 0)) {
    iter++;
    norm[1] = norm[0];
    alpha[1] = alpha[0];
    beta[1] = beta[0];
    omega[1] = omega[0];
    rho[3] = rho[2];
    rho[2] = rho[1];
    rho[1] = mlDot(rt, r);
    if (rho[1] == 0.0) {
      mlIncr(phi, e, 1.0);
      out.finalResidual = norm[0];
      out.exitStatus = 2;
      out.iterations = iter;
      sp_ = saved;
      return out;
    }
    if (init) {
      mlAssign(pv, r);
      init = false;
    } else {
      beta[1] = (rho[1] / rho[2]) * (alpha[1] / omega[1]);
      mlScale(pv, beta[1]);
      mlIncr(pv, v, -beta[1] * omega[1]);
      mlIncr(pv, r, 1.0);
    }
    mlPreCond(pt, pv, p);
    mlZero(v);
    mlApplyOp(v, pt);
    const double m = mlDot(rt, v);
    alpha[0] = rho[1] / m;
    if (std::fabs(m) > p.small * std::fabs(rho[1])) {
      mlIncr(r, v, -alpha[0]);
      norm[0] = mlNorm(r);
      mlIncr(e, pt, alpha[0]);
    } else {
      mlZero(r);
      norm[0] = 0.0;
    }
    out.finalResidual = norm[0];
    if (norm[0] > p.eps * initial_norm && norm[0] > p.reps * out.initialResidual) {
      mlPreCond(st, r, p);
      mlZero(t);
      mlApplyOp(t, st);
      const double tr = mlDot(t, r);
      const double tt = mlDot(t, t);
      omega[0] = tr / tt;
      mlIncr(e, st, omega[0]);
      mlIncr(r, t, -omega[0]);
      norm[0] = mlNorm(r);
    }
    out.finalResidual = norm[0];
    out.history.push_back(norm[0]);
    if (norm[0] <= p.eps * initial_norm || norm[0] <= p.reps * out.initialResidual) {
      out.exitStatus = 1;
      break;
    }
    if (omega[0] == 0.0 || norm[0] > (1 - p.hang) * norm[1]) {
      if (recount == 0) {
        recount = 1;
      } else {
        recount = 0;
        mlIncr(phi, e, 1.0);
        if (restarts == p.numRestarts) {
          out.exitStatus = 3;
          out.iterations = iter;
          sp_ = saved;
          return out;
        }
        mlResidual(r, phi, rhs);
        norm[0] = mlNorm(r);
        rho[1] = 0.0;
        rho[2] = 0.0;
        rho[3] = 0.0;
        alpha[0] = 0;
        beta[0] = 0;
        omega[0] = 0;
        mlAssign(rt, r);
        mlZero(e);
        restarts++;
        init = true;
      }
    }
  }
  out.iterations = iter;
  mlIncr(phi, e, 1.0);
  ck(cudaStreamSynchronize(s_), "bicgstab sync");
  sp_ = saved;
  return out;
}

double Solver::residualNorm() {
  needSingle();
  int lmax = numLevels() - 1;
  std::vector<double*> res(lmax + 1), phi(lmax + 1), rhs(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    res[l] = lev_[l].res;
    phi[l] = lev_[l].phi;
    rhs[l] = lev_[l].rhs;
  }
  return computeAMRResidual(res, phi, rhs, lmax);
}

// AMRMultiGrid::solve -> solveNoInitResid (AMRMultiGrid.H:894-1124).
SolveResult Solver::solve(const SolveParams& p, bool zeroPhi) { return solveImpl(p, zeroPhi, false); }

// Iterative refinement: the FP64 residual of the FP64 phi drives one FP32
// AMR V-cycle per iteration (its input rounded to FP32), whose correction is
// added to phi in FP64; the stopping rules, norms and residual history are
// those of solve().
SolveResult Solver::solveMixed(const SolveParams& p, bool zeroPhi) { return solveImpl(p, zeroPhi, true); }

// One iteration's device work after the norm check: the V-cycle, the update
// of phi and the composite residual with its max-norm (into dNorm_).
void Solver::iterationBody(bool mixed, std::vector<double*>& ures, std::vector<double*>& phi,
                           std::vector<double*>& rhs) {
  const int lmax = numLevels() - 1;
  // A forest changes phi only for the hierarchies still iterating (dActive_).
  const bool forest = nh_ > 1;
  if (!mixed) {
    amrVCycle<double>(lmax, lmax);
    for (int l = 0; l <= lmax; ++l) {
      if (forest)
        incrActive(amrDev_[l], lev_[l].phi, (const double*)lev_[l].ucorr, dActive_, s_);
      else
        incrZero(amrDev_[l], lev_[l].phi, lev_[l].ucorr, s_);  // phi += ucorr; ucorr = 0
      if (forest) zeroField(amrDev_[l], lev_[l].ucorr);
    }
  } else {
    for (int l = 0; l <= lmax; ++l) {
      convert(lev32_[l].ures, lev_[l].ures, amrDev_[l].nelem, s_);
      zeroField(amrDev_[l], lev32_[l].ucorr);
    }
    amrVCycle<float>(lmax, lmax);
    for (int l = 0; l <= lmax; ++l) {
      if (forest)
        incrActive(amrDev_[l], lev_[l].phi, (const float*)lev32_[l].ucorr, dActive_, s_);
      else
        incrMixed(amrDev_[l], lev_[l].phi, lev32_[l].ucorr, s_);
    }
  }
  launchAMRResidual(ures, phi, rhs, lmax);
}

SolveResult Solver::solveImpl(const SolveParams& p, bool zeroPhi, bool mixed) {
  needSingle();
  if (!tuned_) tuneRelaxation();
  if (mixed) ensure32();
  sp_ = p;
  const int lmax = numLevels() - 1;
  SolveResult out;
  std::vector<double*> ures(lmax + 1), phi(lmax + 1), rhs(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    zeroField(amrDev_[l], lev_[l].ucorr);
    zeroField(amrDev_[l], lev_[l].ures);
    if (zeroPhi) zeroField(amrDev_[l], lev_[l].phi);
    ures[l] = lev_[l].ures;
    phi[l] = lev_[l].phi;
    rhs[l] = lev_[l].rhs;
  }
  const double r0 = computeAMRResidual(ures, phi, rhs, lmax);
  double rnorm = r0, normLast = 2 * r0;
  // setConvergenceMetrics(m_initial_rnorm, cushion * m_eps) of the bottom solver
  hostScalars_[1] = r0;
  ck(cudaMemcpyAsync(dMetric_, &hostScalars_[1], sizeof(double), cudaMemcpyHostToDevice, s_), "metric");
  out.history.push_back(rnorm);
  int iter = 0;
  bool goNorm = rnorm > p.normThresh;
  bool goRedu = rnorm > p.eps * r0;
  bool goIter = iter < p.iterMax;
  bool goHang = iter < p.imin || rnorm < (1 - p.hang) * normLast;
  bool goMin = iter < p.iterMin;
  // A NaN or infinite norm ends the solve (the reference's loop stops at a
  // NaN too, since every comparison with it is false); the stopping flags
  // and exit status are computed as for any other norm.
  bool finite = std::isfinite(rnorm);
  const bool graph = useGraphs_ && !profOn_;
  if (p.interrupt) out.interrupted = p.interrupt(0);
  while (finite && !out.interrupted && (goMin || (goIter && goRedu && goHang && goNorm))) {
    normLast = rnorm;
    if (graph) {
      cudaGraphExec_t exec = iterationGraph(mixed, ures, phi, rhs);
      ck(cudaGraphLaunch(exec, s_), "graph launch");
      addLaunches(graphLaunches_[exec]);
    } else {
      iterationBody(mixed, ures, phi, rhs);
    }
    rnorm = readNorm();
    iter++;
    out.history.push_back(rnorm);
    goNorm = rnorm > p.normThresh;
    goRedu = rnorm > p.eps * r0;
    goIter = iter < p.iterMax;
    goHang = iter < p.imin || rnorm < (1 - p.hang) * normLast;
    goMin = iter < p.iterMin;
    finite = std::isfinite(rnorm);
    if (p.interrupt) out.interrupted = p.interrupt(iter);
  }
  out.exitStatus = int(!goRedu) + int(!goIter) * 2 + int(!goHang) * 4 + int(!goNorm) * 8;
  out.iterations = iter;
  out.diverged = !finite;
  return out;
}

// AMRMultiGrid::solve for every hierarchy of a forest together: the loop of
// solveImpl with one norm, stopping rule and iteration count per hierarchy;
// an iteration runs while any hierarchy goes on, and only the going ones
// take its correction.
std::vector<SolveResult> Solver::solveForest(const SolveParams& p, bool zeroPhi, bool mixed,
                                             const std::vector<double>* epsPer,
                                             const std::vector<std::function<int(int)>>* interrupts) {
  if (!tuned_) tuneRelaxation();
  if (mixed) ensure32();
  sp_ = p;
  const int lmax = numLevels() - 1, K = nh_;
  std::vector<SolveResult> out(K);
  std::vector<double*> ures(lmax + 1), phi(lmax + 1), rhs(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    zeroField(amrDev_[l], lev_[l].ucorr);
    zeroField(amrDev_[l], lev_[l].ures);
    if (zeroPhi) zeroField(amrDev_[l], lev_[l].phi);
    ures[l] = lev_[l].ures;
    phi[l] = lev_[l].phi;
    rhs[l] = lev_[l].rhs;
  }
  launchAMRResidual(ures, phi, rhs, lmax);
  const std::vector<double> r0 = readNorms();
  std::vector<double> rnorm = r0, normLast(K);
  if (epsPer && (int)epsPer->size() != K) throw std::invalid_argument("cmg: one tolerance per hierarchy");
  if (interrupts && (int)interrupts->size() != K) throw std::invalid_argument("cmg: one interrupt per hierarchy");
  auto epsOf = [&](int k) { return epsPer ? (*epsPer)[k] : p.eps; };
  // each hierarchy's bottom solver gets its own initial norm as its metric,
  // and its own tolerance
  for (int k = 0; k < K; ++k) {
    hostScalars_[2 + k] = r0[k];
    hostScalars_[2 + K + k] = epsOf(k);
  }
  ck(cudaMemcpyAsync(dMetric_, hostScalars_ + 2, K * sizeof(double), cudaMemcpyHostToDevice, s_), "metric");
  if (K > 1)
    ck(cudaMemcpyAsync(dEps_, hostScalars_ + 2 + K, K * sizeof(double), cudaMemcpyHostToDevice, s_), "tolerances");
  std::vector<char> goNorm(K), goRedu(K), goIter(K), goHang(K), goMin(K), finite(K), going(K);
  std::vector<int> own(K, 0);  // a hierarchy's own interrupt code
  int interrupted = 0;
  auto update = [&](int k, int iter) {
    goNorm[k] = rnorm[k] > p.normThresh;
    goRedu[k] = rnorm[k] > epsOf(k) * r0[k];
    goIter[k] = iter < p.iterMax;
    goHang[k] = iter < p.imin || rnorm[k] < (1 - p.hang) * normLast[k];
    goMin[k] = iter < p.iterMin;
    finite[k] = std::isfinite(rnorm[k]);
    going[k] = finite[k] && !interrupted && !own[k] && (goMin[k] || (goIter[k] && goRedu[k] && goHang[k] && goNorm[k]));
  };
  auto poll = [&](int iter) {
    if (p.interrupt && !interrupted) interrupted = p.interrupt(iter);
    if (interrupts)
      for (int k = 0; k < K; ++k)
        if (!own[k] && (iter == 0 || going[k]) && (*interrupts)[k]) own[k] = (*interrupts)[k](iter);
  };
  poll(0);
  for (int k = 0; k < K; ++k) {
    normLast[k] = 2 * r0[k];
    out[k].history.push_back(rnorm[k]);
    update(k, 0);
  }
  const bool graph = useGraphs_ && !profOn_;
  int iter = 0;
  while (std::any_of(going.begin(), going.end(), [](char g) { return g != 0; })) {
    for (int k = 0; k < K; ++k) {
      hostActive_[k] = going[k];
      if (going[k]) normLast[k] = rnorm[k];
    }
    ck(cudaMemcpyAsync(dActive_, hostActive_, K * sizeof(int), cudaMemcpyHostToDevice, s_), "active flags");
    if (graph) {
      cudaGraphExec_t exec = iterationGraph(mixed, ures, phi, rhs);
      ck(cudaGraphLaunch(exec, s_), "graph launch");
      addLaunches(graphLaunches_[exec]);
    } else {
      iterationBody(mixed, ures, phi, rhs);
    }
    const std::vector<double> r = readNorms();
    iter++;
    poll(iter);
    for (int k = 0; k < K; ++k) {
      if (!hostActive_[k]) continue;
      rnorm[k] = r[k];
      out[k].iterations = iter;
      out[k].history.push_back(rnorm[k]);
      update(k, iter);
    }
  }
  for (int k = 0; k < K; ++k) {
    out[k].exitStatus = int(!goRedu[k]) + int(!goIter[k]) * 2 + int(!goHang[k]) * 4 + int(!goNorm[k]) * 8;
    out[k].diverged = !finite[k];
    out[k].interrupted = own[k] ? own[k] : interrupted;
  }
  return out;
}

// The iteration body captured once per (precision, smoothing parameters)
// into a CUDA graph and replayed: every pointer and launch argument of the
// body is fixed for the hierarchy; the bottom solver's metric is read from
// device memory at run time.
cudaGraphExec_t Solver::iterationGraph(bool mixed, std::vector<double*>& ures, std::vector<double*>& phi,
                                       std::vector<double*>& rhs) {
  GraphKey key{mixed, sp_.pre, sp_.post, sp_.bottom, sp_.numMG, sp_.eps, desc_.alpha, desc_.beta};
  auto it = graphs_.find(key);
  if (it != graphs_.end()) return it->second;
  if (graphs_.size() >= kMaxGraphs) {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
  }
  cudaGraph_t g = nullptr;
  const long long before = launchCount();
  ck(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    iterationBody(mixed, ures, phi, rhs);
  } catch (...) {
    cudaStreamEndCapture(s_, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  ck(cudaStreamEndCapture(s_, &g), "end capture");
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  ck(e, "graph instantiate");
  graphs_[key] = exec;
  // the captured launches did not run; each replay adds them
  graphLaunches_[exec] = launchCount() - before;
  addLaunches(-(launchCount() - before));
  return exec;
}

void Solver::setUseGraphs(bool on) { useGraphs_ = on; }

float* Solver::allocF(size_t n) {
  bufs_.emplace_back(new DevBuf(n * sizeof(float), own_));
  ownSync();
  float* p = (float*)bufs_.back()->p;
  ck(cudaMemsetAsync(p, 0, n * sizeof(float), s_), "memset");
  return p;
}

void Solver::ensure32() {
  if (!have32_) {
    lev32_.resize(amr_.size());
    for (size_t l = 0; l < amr_.size(); ++l) {
      const size_t n = amr_[l].nelem;
      FieldsT<float>& f = lev32_[l];
      f.ures = allocF(n);
      f.ucorr = allocF(n);
      f.corr = allocF(n);
      f.res = allocF(n);
      if (desc_.vc) {
        f.a = allocF(n);
        for (int d = 0; d < 3; ++d) f.b[d] = allocF(n);
        f.lambda = allocF(n);
      }
    }
    mgf32_.resize(mg_.size());
    for (size_t d = 0; d < mg_.size(); ++d) {
      const size_t n = mg_[d].nelem;
      FieldsT<float>& f = mgf32_[d];
      f.corr = allocF(n);
      f.res = allocF(n);
      if (desc_.vc) {
        f.a = allocF(n);
        for (int k = 0; k < 3; ++k) f.b[k] = allocF(n);
        f.lambda = allocF(n);
      }
    }
    have32_ = true;
    coef32Stale_ = true;
  }
  if (desc_.vc && coef32Stale_) {
    // The FP32 operators use the FP64 coefficients (and relaxation
    // coefficient) rounded to FP32.
    for (size_t l = 0; l < amr_.size(); ++l) {
      const int64_t n = amr_[l].nelem;
      convert(lev32_[l].a, lev_[l].a, n, s_);
      for (int d = 0; d < 3; ++d) convert(lev32_[l].b[d], lev_[l].b[d], n, s_);
      convert(lev32_[l].lambda, lev_[l].lambda, n, s_);
    }
    for (size_t d = 0; d < mg_.size(); ++d) {
      const int64_t n = mg_[d].nelem;
      convert(mgf32_[d].a, mgf_[d].a, n, s_);
      for (int k = 0; k < 3; ++k) convert(mgf32_[d].b[k], mgf_[d].b[k], n, s_);
      convert(mgf32_[d].lambda, mgf_[d].lambda, n, s_);
    }
    coef32Stale_ = false;
  }
}

double Solver::vcycleBytes(const SolveParams& p) const {
  // Per valid cell, in FP64 words: one GSRB colour pass reads phi and half of
  // rhs and writes half of phi (VC adds half a, half lambda, all b faces);
  // residual/operator passes read phi, rhs and write one array.
  const double s = 8.0;
  const double vc = desc_.vc ? 1.0 : 0.0;
  const double colour = 2.0 + vc * 4.0;
  const double resid = 3.0 + vc * 4.0;
  double total = 0;
  for (int l = 0; l < numLevels(); ++l) {
    double n = (double)amr_[l].grids.numCells();
    double sweeps = l == 0 && numLevels() == 1 ? p.pre + p.post : p.pre + p.post;
    total += n * s * (2 * sweeps * colour + 3 * resid);
  }
  for (size_t d = 0; d < mg_.size(); ++d) {
    double n = (double)mg_[d].grids.numCells();
    total += n * s * (2 * (p.pre + p.post) * colour + resid);
  }
  return total;
}

}  // namespace cmg

namespace cmg {

cudaEvent_t Solver::takeEvent() {
  if (!evPool_.empty()) {
    cudaEvent_t e = evPool_.back();
    evPool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  ck(cudaEventCreate(&e), "event");
  return e;
}

void Solver::profileDrain() {
  if (prof_.empty()) return;
  ck(cudaStreamSynchronize(s_), "profile sync");
  for (const ProfRec& r : prof_) {
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, r.a, r.b), "event elapsed");
    profAcc_[r.cls][0] += 1;
    profAcc_[r.cls][1] += ms;
    profAcc_[r.cls][2] += r.bytes;
    evPool_.push_back(r.a);
    evPool_.push_back(r.b);
  }
  prof_.clear();
}

void Solver::profileEnable(bool on) {
  profileDrain();
  profOn_ = on;
  for (auto& c : profAcc_) c[0] = c[1] = c[2] = 0;
}

void Solver::profileRead(int cls, int64_t* launches, double* ms, double* bytes) {
  if (cls < 0 || cls >= P_NCLASS) throw std::invalid_argument("cmg: profile class out of range");
  profileDrain();
  *launches = (int64_t)profAcc_[cls][0];
  *ms = profAcc_[cls][1];
  *bytes = profAcc_[cls][2];
}

}  // namespace cmg
