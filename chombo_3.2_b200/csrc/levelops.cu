// Operator-level calls: one method of AMRLevelOp / MGLevelOp / LinearOp
// (AMRElliptic/AMRMultiGrid.H:39-225, MultiGrid.H:116-160,
// LinearSolver.H:41-137) of one level of a hierarchy, as AMRPoissonOp and
// VCAMRPoissonOp2 implement them, on host arrays.  This is what a Chombo
// program's own AMRMultiGrid, MultiGrid or BiCGStabSolver calls when it
// drives the GPU operators one virtual at a time (the AMRLevelOp drop-in of
// include/cmg_chombo.H).  Every call moves its arguments to the level's
// device layout, runs the same kernels as the device-resident solve, and
// moves the outputs back.
//
// Host array format ("ghosted"): every box's FAB grown by one cell (the
// reference's phi layout, ghost 1, one component), x fastest, boxes in layout
// order.  Inputs are read in full (ghost positions included: an operator
// that does not refill a ghost cell reads the caller's value, as the
// reference reads whatever its FAB holds).  Outputs get their valid cells
// written; their ghost positions are unspecified.
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "solver.H"

namespace cmg {

namespace {

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "cmg: %s: %s", what, cudaGetErrorString(e));
    throw std::runtime_error(buf);
  }
}

// Ghosted host format <-> device layout, one block per box.  mode 1: every
// cell of the grown box is written to the device; mode 0: the valid cells
// are written to the host-format buffer; mode 2: every grown-box cell is.
__global__ void k_ghosted(const BoxDesc* boxes, const int64_t* off, double* dev, double* buf, int toDev) {
  const BoxDesc b = boxes[blockIdx.x];
  const int gx = b.hi[0] - b.lo[0] + 3, gy = b.hi[1] - b.lo[1] + 3, gz = b.hi[2] - b.lo[2] + 3;
  const int64_t o = off[blockIdx.x];
  if (toDev == 2) {
    for (int q = threadIdx.x; q < gx * gy * gz; q += blockDim.x) {
      const int i = q % gx, t = q / gx, j = t % gy, k = t / gy;
      buf[o + q] = dev[cellIndex(b, b.lo[0] - 1 + i, b.lo[1] - 1 + j, b.lo[2] - 1 + k)];
    }
  } else if (toDev) {
    for (int q = threadIdx.x; q < gx * gy * gz; q += blockDim.x) {
      const int i = q % gx, t = q / gx, j = t % gy, k = t / gy;
      dev[cellIndex(b, b.lo[0] - 1 + i, b.lo[1] - 1 + j, b.lo[2] - 1 + k)] = buf[o + q];
    }
  } else {
    const int nx = gx - 2, ny = gy - 2, nz = gz - 2;
    for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
      const int i = q % nx, t = q / nx, j = t % ny, k = t / ny;
      buf[o + (i + 1) + (int64_t)gx * ((j + 1) + (int64_t)gy * (k + 1))] =
          dev[cellIndex(b, b.lo[0] + i, b.lo[1] + j, b.lo[2] + k)];
    }
  }
}

// FORT_AVERAGE with refRatio 2 (AMRTools/AverageF.ChF:36-55) of fine box b
// into coarsen(box b) of the coarsened-fine layout, written in the ghosted
// host format (AMRPoissonOp::AMRRestrictS, AMRPoissonOp.cpp:877-919).
__global__ void k_average_cfine(const BoxDesc* fboxes, const int64_t* coff, const double* fine, double* out) {
  const BoxDesc fb = fboxes[blockIdx.x];
  const int clo[3] = {fb.lo[0] >> 1, fb.lo[1] >> 1, fb.lo[2] >> 1};
  const int nx = ((fb.hi[0] + 1) >> 1) - clo[0], ny = ((fb.hi[1] + 1) >> 1) - clo[1],
            nz = ((fb.hi[2] + 1) >> 1) - clo[2];
  const int64_t o = coff[blockIdx.x];
  for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
    const int a = q % nx, t = q / nx, c = t % ny, e = t / ny;
    const int i = 2 * (clo[0] + a), j = 2 * (clo[1] + c), k = 2 * (clo[2] + e);
    double sum = fine[cellIndex(fb, i, j, k)] + fine[cellIndex(fb, i + 1, j, k)] + fine[cellIndex(fb, i, j + 1, k)] +
                 fine[cellIndex(fb, i + 1, j + 1, k)] + fine[cellIndex(fb, i, j, k + 1)] +
                 fine[cellIndex(fb, i + 1, j, k + 1)] + fine[cellIndex(fb, i, j + 1, k + 1)] +
                 fine[cellIndex(fb, i + 1, j + 1, k + 1)];
    out[o + (a + 1) + (int64_t)(nx + 2) * ((c + 1) + (int64_t)(ny + 2) * (e + 1))] = 0.125 * sum;
  }
}

// AMRMultiGrid's assignCopier from the coarsened-fine layout into the coarse
// level (AMRMultiGrid.H:1391, Copier m_resCopier): every coarse valid cell
// under a fine box takes the coarsened-fine value, through the coarse/fine
// items of the fine level (region in coarse index space).
__global__ void k_assign_cfine(const CoarseFineItem* items, const BoxDesc* fboxes, const BoxDesc* cboxes,
                               const int64_t* coff, const double* in, double* coarse) {
  const CoarseFineItem it = items[blockIdx.x];
  const BoxDesc fb = fboxes[it.fbox];
  const int clo[3] = {fb.lo[0] >> 1, fb.lo[1] >> 1, fb.lo[2] >> 1};
  const int cnx = ((fb.hi[0] + 1) >> 1) - clo[0], cny = ((fb.hi[1] + 1) >> 1) - clo[1];
  const int nx = it.hi[0] - it.lo[0] + 1, ny = it.hi[1] - it.lo[1] + 1, nz = it.hi[2] - it.lo[2] + 1;
  const int64_t o = coff[it.fbox];
  for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
    const int I = it.lo[0] + q % nx, t = q / nx, J = it.lo[1] + t % ny, K = it.lo[2] + t / ny;
    coarse[cellIndex(cboxes[it.cbox], I, J, K)] =
        in[o + (I - clo[0] + 1) + (int64_t)(cnx + 2) * ((J - clo[1] + 1) + (int64_t)(cny + 2) * (K - clo[2] + 1))];
  }
}

// AMRPoissonOp::preCond / VCAMRPoissonOp2::preCond (AMRPoissonOp.cpp:304-329,
// VCAMRPoissonOp2.cpp:93-127): phi = rhs * mult, or rhs * lambda, valid cells.
__global__ void k_precond(const BoxDesc* boxes, const Chunk* chunks, double* cor, const double* res,
                          const double* lam, double mult) {
  const Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1, nz = bd.hi[2] - bd.lo[2] + 1;
  const int q = ch.start + threadIdx.x;
  if (q >= nx * ny * nz) return;
  const int i = bd.lo[0] + q % nx, t = q / nx, j = bd.lo[1] + t % ny, k = bd.lo[2] + t / ny;
  const int64_t c = cellIndex(bd, i, j, k);
  cor[c] = lam ? res[c] * lam[c] : res[c] * mult;
}

// LevelDataOps::axby (LevelDataOps.H:255-268: lhs = x; lhs *= a; lhs += y*b),
// ::incr (lhs += x*scale) and ::scale (lhs *= scale), element by element of
// the ghosted host format (valid cells are what the caller keeps).
__global__ void k_axby_flat(double* lhs, const double* x, const double* y, double a, double b, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    double v = x[q] * a;
    lhs[q] = v + y[q] * b;
  }
}
__global__ void k_incr_packed(double* lhs, const double* x, double s, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    lhs[q] = lhs[q] + x[q] * s;
}
__global__ void k_scale_packed(double* lhs, double s, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    lhs[q] = lhs[q] * s;
}

// FArrayBox::norm(p = 1) and sumPow(p = 2) of one box's valid cells
// (BoxTools/FArrayBox.cpp:62-209): per x position, a running value over the
// box's pencils in (k, j) order, then the positions summed in x order.  One
// block per box; positions are spread over the threads, the final sum is
// taken by thread 0.
__global__ void k_box_pencil(const BoxDesc* boxes, const double* x, int p, double* out) {
  extern __shared__ double tmp[];
  const BoxDesc b = boxes[blockIdx.x];
  const int nx = b.hi[0] - b.lo[0] + 1;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    double acc = 0.0;
    bool first = true;
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
      for (int j = b.lo[1]; j <= b.hi[1]; ++j) {
        const double v = x[cellIndex(b, b.lo[0] + i, j, k)];
        const double w = p == 1 ? fabs(v) : v * v;
        acc = first ? w : acc + w;
        first = false;
      }
    tmp[i] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = tmp[0];
    for (int i = 1; i < nx; ++i) s += tmp[i];
    out[blockIdx.x] = s;
  }
}

// FArrayBox::norm(p = 0) of one box: max |x| over the valid cells; a NaN
// anywhere makes the box's value NaN.
__global__ void k_box_absmax(const BoxDesc* boxes, const double* x, double* out) {
  __shared__ double red[32];
  const BoxDesc b = boxes[blockIdx.x];
  const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
  double m = 0.0;
  for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
    const int i = q % nx, t = q / nx, j = t % ny, k = t / ny;
    const double v = fabs(x[cellIndex(b, b.lo[0] + i, b.lo[1] + j, b.lo[2] + k)]);
    m = (v > m || v != v) ? v : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, m, o);
    m = (w > m || w != w) ? w : m;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = (red[w] > r || red[w] != red[w]) ? red[w] : r;
    out[blockIdx.x] = r;
  }
}

inline int flatGrid(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 8); }

}  // namespace

// ------------------------------------------------------------ level access

const LevelPlan& Solver::opPlan(int lev) const {
  if (lev >= 0) {
    if (lev >= numLevels()) throw std::invalid_argument("cmg: level out of range");
    return amr_[lev];
  }
  if (-lev > (int)mg_.size()) throw std::invalid_argument("cmg: multigrid depth out of range");
  return mg_[-lev - 1];
}

const LevelDev& Solver::opDev(int lev) const { return lev >= 0 ? amrDev_[lev] : mgDev_[-lev - 1]; }

Coef<double> Solver::opCoef(int lev) const { return lev >= 0 ? coefAMR(lev) : coefMG(-lev); }

int64_t Solver::opSize(int lev) const {
  int64_t n = 0;
  for (const Box& b : opPlan(lev).grids.boxes) n += b.grow(1).numPts();
  return n;
}

int64_t Solver::opCoarsenedSize(int l) const {
  if (l < 1 || l >= numLevels()) throw std::invalid_argument("cmg: coarsened layout needs a level >= 1");
  int64_t n = 0;
  for (const Box& b : amr_[l].grids.boxes) n += b.coarsen(2).grow(1).numPts();
  return n;
}

// Device-side state of the operator calls of one level: offsets of every box
// in the ghosted host format (and, for AMR levels >= 1, in the coarsened-fine
// format), a host staging buffer, and level-sized device fields.
Solver::OpState& Solver::opState(int lev) {
  needSingle();
  auto it = opStates_.find(lev);
  if (it != opStates_.end()) return *it->second;
  const LevelPlan& p = opPlan(lev);
  std::unique_ptr<OpState> st(new OpState);
  std::vector<int64_t> off, coff;
  int64_t n = 0, nc = 0;
  for (const Box& b : p.grids.boxes) {
    off.push_back(n);
    n += b.grow(1).numPts();
    if (lev >= 1) {
      coff.push_back(nc);
      nc += b.coarsen(2).grow(1).numPts();
    }
  }
  st->size = n;
  st->csize = nc;
  st->off = (const int64_t*)uploadRaw(off.data(), off.size() * sizeof(int64_t));
  if (lev >= 1) st->coff = (const int64_t*)uploadRaw(coff.data(), coff.size() * sizeof(int64_t));
  st->packed = alloc(std::max<int64_t>(n, nc));
  st->packed2 = alloc(std::max<int64_t>(n, nc));
  st->packed3 = alloc(std::max<int64_t>(n, nc));
  it = opStates_.emplace(lev, std::move(st)).first;
  return *it->second;
}

double* Solver::opField(int lev, int k) {
  OpState& st = opState(lev);
  if (k < 0 || k >= OpState::kFields) throw std::logic_error("cmg: operator field index");
  if (!st.field[k]) st.field[k] = alloc(opPlan(lev).nelem);
  return st.field[k];
}

void* Solver::uploadRaw(const void* src, size_t bytes) {
  bufs_.emplace_back(new DevBuf(bytes, own_));
  ck(cudaMemcpyAsync(bufs_.back()->p, src, bytes, cudaMemcpyHostToDevice, own_), "upload");
  ck(cudaStreamSynchronize(own_), "upload sync");
  return bufs_.back()->p;
}

// Host ghosted array -> device field k of level lev (every grown-box cell).
double* Solver::opLoad(int lev, int k, const double* host) {
  if (!host) throw std::invalid_argument("cmg: null operator argument");
  OpState& st = opState(lev);
  double* f = opField(lev, k);
  const LevelDev& L = opDev(lev);
  if (L.nbox == 0) return f;
  ck(cudaMemcpyAsync(st.packed, host, st.size * sizeof(double), cudaMemcpyHostToDevice, s_), "operator h2d");
  k_ghosted<<<L.nbox, 256, 0, s_>>>(L.boxes, st.off, f, st.packed, 1);
  ck(cudaGetLastError(), "operator scatter");
  return f;
}

// Valid cells of device field f of level lev -> host ghosted array.
void Solver::opStore(int lev, const double* f, double* host) {
  OpState& st = opState(lev);
  const LevelDev& L = opDev(lev);
  if (L.nbox == 0) return;
  k_ghosted<<<L.nbox, 256, 0, s_>>>(L.boxes, st.off, const_cast<double*>(f), st.packed, 0);
  ck(cudaGetLastError(), "operator gather");
  ck(cudaMemcpyAsync(host, st.packed, st.size * sizeof(double), cudaMemcpyDeviceToHost, s_), "operator d2h");
  ck(cudaStreamSynchronize(s_), "operator sync");
}

// Every cell of device field f of level lev (valid and ghost) -> host
// ghosted array.
void Solver::opStoreGrown(int lev, const double* f, double* host) {
  OpState& st = opState(lev);
  const LevelDev& L = opDev(lev);
  if (L.nbox == 0) return;
  k_ghosted<<<L.nbox, 256, 0, s_>>>(L.boxes, st.off, const_cast<double*>(f), st.packed, 2);
  ck(cudaGetLastError(), "operator gather");
  ck(cudaMemcpyAsync(host, st.packed, st.size * sizeof(double), cudaMemcpyDeviceToHost, s_), "operator d2h");
  ck(cudaStreamSynchronize(s_), "operator sync");
}

void Solver::opEnsureTuned() {
  if (!tuned_) tuneRelaxation();
}

// ------------------------------------------------------------ LinearOp / MGLevelOp

// AMRPoissonOp::residual (AMRPoissonOp.cpp:227-238) -> residualI: a
// homogeneous residual first sets the homogeneous coarse-fine ghosts; then
// exchange and boundary values, and OPERATORLAPRES / VCCOMPUTERES3D.
void Solver::opResidual(int lev, double* lhs, const double* phi, const double* rhs, bool homogeneous) {
  const LevelDev& L = opDev(lev);
  double* f = opLoad(lev, 0, phi);
  double* r = opLoad(lev, 1, rhs);
  double* o = opField(lev, 2);
  ghostFill(L, f, homogeneous && lev > 0, s_);
  residual(L, o, f, r, opCoef(lev), s_);
  opStore(lev, o, lhs);
}

// AMRPoissonOp::applyOp (AMRPoissonOp.cpp:332-341): homogeneous coarse-fine
// ghosts, then applyOpI.
void Solver::opApply(int lev, double* lhs, const double* phi, bool homogeneous) {
  const LevelDev& L = opDev(lev);
  double* f = opLoad(lev, 0, phi);
  double* o = opField(lev, 2);
  ghostFill(L, f, lev > 0, s_);
  (void)homogeneous;  // homogeneous Dirichlet is the only physical boundary condition
  applyOp(L, o, f, opCoef(lev), s_);
  opStore(lev, o, lhs);
}

// AMRPoissonOp::relax (AMRPoissonOp.cpp:600-632): iterations x levelGSRB.
void Solver::opRelax(int lev, double* phi, const double* rhs, int iterations) {
  opEnsureTuned();
  double* f = opLoad(lev, 0, phi);
  double* r = opLoad(lev, 1, rhs);
  if (lev >= 0)
    relaxAMR<double>(lev, f, r, iterations);
  else
    relaxMG<double>(-lev, f, r, iterations);
  opStore(lev, f, phi);
}

// AMRPoissonOp::preCond / VCAMRPoissonOp2::preCond: the inverse diagonal
// times the residual, then two relaxation sweeps.
void Solver::opPreCond(int lev, double* cor, const double* res) {
  opEnsureTuned();
  const LevelDev& L = opDev(lev);
  const Coef<double> c = opCoef(lev);
  double* f = opLoad(lev, 0, cor);
  double* r = opLoad(lev, 1, res);
  const double mult = 1.0 / (c.alpha - 2.0 * 3 * c.beta / (L.dx * L.dx));
  if (L.nAll > 0) {
    k_precond<<<L.nAll, CHUNK, 0, s_>>>(L.boxes, L.chAll, f, r, c.vc ? c.lambda : nullptr, mult);
    ck(cudaGetLastError(), "preCond");
  }
  if (lev >= 0)
    relaxAMR<double>(lev, f, r, 2);
  else
    relaxMG<double>(-lev, f, r, 2);
  opStore(lev, f, cor);
}

// AMRPoissonOp::restrictResidual (AMRPoissonOp.cpp:651-703) and
// VCAMRPoissonOp2::restrictResidual: ghosts, then RESTRICTRES(VC3D) into the
// next multigrid depth.
void Solver::opRestrictResidual(int lev, double* resCoarse, const double* phi, const double* rhs) {
  if (lev > 0) throw std::invalid_argument("cmg: multigrid restriction runs below AMR level 0 only");
  const int clev = lev - 1;
  opPlan(clev);
  const LevelDev& F = opDev(lev);
  double* f = opLoad(lev, 0, phi);
  double* r = opLoad(lev, 1, rhs);
  double* rc = opLoad(clev, 2, resCoarse);
  ghostFill(F, f, false, s_);
  restrictMG(F, opDev(clev), rc, f, r, opCoef(lev), s_);
  opStore(clev, rc, resCoarse);
}

// AMRPoissonOp::prolongIncrement (AMRPoissonOp.cpp:706-733): PROLONG.
void Solver::opProlongIncrement(int lev, double* phi, const double* corrCoarse) {
  if (lev > 0) throw std::invalid_argument("cmg: multigrid prolongation runs below AMR level 0 only");
  const int clev = lev - 1;
  opPlan(clev);
  double* f = opLoad(lev, 0, phi);
  double* c = opLoad(clev, 1, corrCoarse);
  prolongMG(opDev(lev), opDev(clev), f, c, s_);
  opStore(lev, f, phi);
}

// ------------------------------------------------------------ AMRLevelOp

// AMRPoissonOp::AMROperator / AMROperatorNC / AMROperatorNF and the
// AMRResidual family (AMRPoissonOp.cpp:736-858): inhomogeneous coarse-fine
// interpolation from phiCoarse (when given), exchange and boundary values,
// then
//   form 0: out = L(phi)           (applyOpI, plus reflux with phiFine),
//   form 1: out = rhs - L(phi)     (the same, then axby(out, out, rhs, -1, 1)),
//   form 2: out = rhs - L(phi)     (residualI: OPERATORLAPRES / VCCOMPUTERES3D).
void Solver::opAMROperator(int l, double* out, const double* phiFine, double* phi, const double* phiCoarse,
                           const double* rhs, int form) {
  if (l < 0 || l >= numLevels()) throw std::invalid_argument("cmg: AMR level out of range");
  if (phiCoarse && l == 0) throw std::invalid_argument("cmg: level 0 has no coarser level");
  if (phiFine && l + 1 >= numLevels()) throw std::invalid_argument("cmg: no finer level");
  if (form < 0 || form > 2 || (form != 0 && !rhs)) throw std::invalid_argument("cmg: bad operator form");
  if (form == 2 && phiFine) throw std::invalid_argument("cmg: the residualI form has no finer level");
  const LevelDev& L = amrDev_[l];
  double* f = opLoad(l, 0, phi);
  double* r = rhs ? opLoad(l, 1, rhs) : nullptr;
  double* o = opField(l, 2);
  if (phiCoarse) quadCF(L, f, opLoad(l - 1, 3, phiCoarse), s_);
  ghostFill(L, f, false, s_);
  const Coef<double> c = coefAMR(l);
  if (form == 2) {
    residual(L, o, f, r, c, s_);
  } else {
    applyOp(L, o, f, c, s_);
    if (phiFine) {
      double* ff = opLoad(l + 1, 4, phiFine);
      quadCF(amrDev_[l + 1], ff, f, s_);
      reflux(L, o, f, ff, c, coefAMR(l + 1), s_);
    }
    if (form == 1) negAdd(L, o, o, r, s_);
  }
  opStore(l, o, out);
  opStoreGrown(l, f, phi);
}

// AMRPoissonOp::AMRRestrictS (AMRPoissonOp.cpp:877-919): the residual of
// the correction with coarse-fine values from the coarse correction
// (AMRResidualNF, homogeneous physical boundary), averaged onto the
// coarsened-fine layout (ghosted host format of coarsen(box, 2)).
void Solver::opAMRRestrict(int l, double* resCoarsened, const double* residual_, const double* corr,
                           const double* corrCoarse) {
  if (l < 1 || l >= numLevels()) throw std::invalid_argument("cmg: AMR restriction needs a level >= 1");
  const LevelDev& L = amrDev_[l];
  OpState& st = opState(l);
  double* r = opLoad(l, 1, residual_);
  double* s = r;
  if (corr) {
    // AMRResidualNF(scratch, correction, coarseCorrection, residual, true)
    double* e = opLoad(l, 0, corr);
    s = opField(l, 2);
    quadCF(L, e, opLoad(l - 1, 3, corrCoarse), s_);
    ghostFill(L, e, false, s_);
    residual(L, s, e, r, coefAMR(l), s_);
  }  // else a_skip_res: the residual itself is averaged (the FAS restriction of phi)
  if (L.nbox > 0) {
    k_average_cfine<<<L.nbox, 256, 0, s_>>>(L.boxes, st.coff, s, st.packed2);
    ck(cudaGetLastError(), "average");
  }
  ck(cudaMemcpyAsync(resCoarsened, st.packed2, st.csize * sizeof(double), cudaMemcpyDeviceToHost, s_), "d2h");
  ck(cudaStreamSynchronize(s_), "operator sync");
}

// assignCopier(coarse, coarsened) of AMRVCycle (AMRMultiGrid.H:1391): the
// coarsened-fine data of level l copied onto the valid cells of level l - 1
// that level l covers.
void Solver::opAssignCoarsened(int l, double* coarse, const double* coarsened) {
  if (l < 1 || l >= numLevels()) throw std::invalid_argument("cmg: coarsened layout needs a level >= 1");
  OpState& st = opState(l);
  double* c = opLoad(l - 1, 0, coarse);
  ck(cudaMemcpyAsync(st.packed2, coarsened, st.csize * sizeof(double), cudaMemcpyHostToDevice, s_), "h2d");
  const int nitems = (int)amr_[l].toCoarse.size();
  if (nitems > 0) {
    k_assign_cfine<<<nitems, 256, 0, s_>>>(amrDev_[l].items, amrDev_[l].boxes, amrDev_[l - 1].boxes, st.coff,
                                            st.packed2, c);
    ck(cudaGetLastError(), "assign coarsened");
  }
  opStore(l - 1, c, coarse);
}

// AMRPoissonOp::AMRProlongS / AMRProlong (AMRPoissonOp.cpp:926-990):
// correction += coarse correction at the parent cell.
void Solver::opAMRProlong(int l, double* corr, const double* corrCoarse) {
  if (l < 1 || l >= numLevels()) throw std::invalid_argument("cmg: AMR prolongation needs a level >= 1");
  double* e = opLoad(l, 0, corr);
  double* c = opLoad(l - 1, 1, corrCoarse);
  prolongAMR(amrDev_[l], amrDev_[l - 1], e, c, s_);
  opStore(l, e, corr);
}

// AMRPoissonOp::AMRUpdateResidual (AMRPoissonOp.cpp:1045-1054):
// AMRResidualNF(residual, correction, coarseCorrection, residual, true).
void Solver::opAMRUpdateResidual(int l, double* res, const double* corr, const double* corrCoarse) {
  if (l < 1 || l >= numLevels()) throw std::invalid_argument("cmg: residual update needs a level >= 1");
  const LevelDev& L = amrDev_[l];
  double* e = opLoad(l, 0, corr);
  double* r = opLoad(l, 1, res);
  quadCF(L, e, opLoad(l - 1, 3, corrCoarse), s_);
  ghostFill(L, e, false, s_);
  residual(L, r, e, r, coefAMR(l), s_);
  opStore(l, r, res);
}

// QuadCFInterp::coarseFineInterp (AMRTools/QuadCFInterp.cpp:845-889): the
// coarse-fine face ghosts of phi on level l from phiCoarse; phi comes back
// whole (valid and ghost cells).
void Solver::opCFInterp(int l, double* phi, const double* phiCoarse) {
  if (l < 1 || l >= numLevels()) throw std::invalid_argument("cmg: coarse-fine interpolation needs a level >= 1");
  double* f = opLoad(l, 0, phi);
  quadCF(amrDev_[l], f, opLoad(l - 1, 3, phiCoarse), s_);
  opStoreGrown(l, f, phi);
}

// AMRLevelOp::zeroCovered (AMRMultiGrid.H:197-201): the valid cells of level
// l under level l + 1 set to zero.
void Solver::opZeroCovered(int l, double* data) {
  if (l < 0 || l + 1 >= numLevels()) throw std::invalid_argument("cmg: zeroCovered needs a finer level");
  double* f = opLoad(l, 0, data);
  zeroCovered(amrDev_[l], f, s_);
  opStore(l, f, data);
}

// ------------------------------------------------------------ LevelDataOps

void Solver::opAxby(int lev, double* lhs, const double* x, const double* y, double a, double b) {
  OpState& st = opState(lev);
  const int64_t n = st.size;
  if (n == 0) return;
  ck(cudaMemcpyAsync(st.packed2, x, n * sizeof(double), cudaMemcpyHostToDevice, s_), "h2d");
  ck(cudaMemcpyAsync(st.packed3, y, n * sizeof(double), cudaMemcpyHostToDevice, s_), "h2d");
  k_axby_flat<<<flatGrid(n), 256, 0, s_>>>(st.packed, st.packed2, st.packed3, a, b, n);
  ck(cudaGetLastError(), "axby");
  ck(cudaMemcpyAsync(lhs, st.packed, n * sizeof(double), cudaMemcpyDeviceToHost, s_), "d2h");
  ck(cudaStreamSynchronize(s_), "operator sync");
}

void Solver::opIncr(int lev, double* lhs, const double* x, double scale) {
  OpState& st = opState(lev);
  const int64_t n = st.size;
  if (n == 0) return;
  ck(cudaMemcpyAsync(st.packed, lhs, n * sizeof(double), cudaMemcpyHostToDevice, s_), "h2d");
  ck(cudaMemcpyAsync(st.packed2, x, n * sizeof(double), cudaMemcpyHostToDevice, s_), "h2d");
  k_incr_packed<<<flatGrid(n), 256, 0, s_>>>(st.packed, st.packed2, scale, n);
  ck(cudaGetLastError(), "incr");
  ck(cudaMemcpyAsync(lhs, st.packed, n * sizeof(double), cudaMemcpyDeviceToHost, s_), "d2h");
  ck(cudaStreamSynchronize(s_), "operator sync");
}

void Solver::opScale(int lev, double* lhs, double scale) {
  OpState& st = opState(lev);
  const int64_t n = st.size;
  if (n == 0) return;
  ck(cudaMemcpyAsync(st.packed, lhs, n * sizeof(double), cudaMemcpyHostToDevice, s_), "h2d");
  k_scale_packed<<<flatGrid(n), 256, 0, s_>>>(st.packed, scale, n);
  ck(cudaGetLastError(), "scale");
  ck(cudaMemcpyAsync(lhs, st.packed, n * sizeof(double), cudaMemcpyDeviceToHost, s_), "d2h");
  ck(cudaStreamSynchronize(s_), "operator sync");
}

// Per-box values read back and combined in box order on the host, as the
// reference's loops over the DataIterator do.
std::vector<double> Solver::opBoxValues(int lev, int nbox) {
  std::vector<double> v(nbox);
  if (nbox == 0) return v;
  OpState& st = opState(lev);
  ck(cudaMemcpyAsync(v.data(), st.packed2, nbox * sizeof(double), cudaMemcpyDeviceToHost, s_), "d2h");
  ck(cudaStreamSynchronize(s_), "operator sync");
  return v;
}

// LevelDataOps::dotProduct (LevelDataOps.H:109-131): FArrayBox::dotProduct
// of every box (k, j, i order, i fastest), summed in box order from zero.
double Solver::opDot(int lev, const double* x, const double* y) {
  const LevelDev& L = opDev(lev);
  double* a = opLoad(lev, 0, x);
  double* b = opLoad(lev, 1, y);
  OpState& st = opState(lev);
  boxDots(L, a, b, st.packed2, s_);
  double val = 0;
  for (double v : opBoxValues(lev, L.nbox)) val += v;
  return val;
}

// norm(BoxLayoutData, interval, p) (BoxTools/BoxLayoutData.cpp:23-93) as
// AMRPoissonOp::norm calls it: p = 0 the max over boxes of FArrayBox::norm,
// p = 1 the sum of the boxes' norms, otherwise the sum of the boxes' sumPow,
// then its p-th root (sqrt for p = 2).
double Solver::opNorm(int lev, const double* x, int p) {
  if (p < 0 || p > 2) throw std::invalid_argument("cmg: norm order is 0, 1 or 2");
  const LevelDev& L = opDev(lev);
  double* a = opLoad(lev, 0, x);
  OpState& st = opState(lev);
  if (L.nbox == 0) return 0.0;
  if (p == 0) {
    k_box_absmax<<<L.nbox, 256, 0, s_>>>(L.boxes, a, st.packed2);
  } else {
    int maxnx = 1;
    for (const Box& b : opPlan(lev).grids.boxes) maxnx = std::max(maxnx, b.hi[0] - b.lo[0] + 1);
    if (maxnx * sizeof(double) > 48 * 1024) throw std::invalid_argument("cmg: box too wide for the norm kernel");
    k_box_pencil<<<L.nbox, 128, maxnx * sizeof(double), s_>>>(L.boxes, a, p, st.packed2);
  }
  ck(cudaGetLastError(), "norm");
  const std::vector<double> v = opBoxValues(lev, L.nbox);
  double norm = 0;
  if (p == 0) {
    // Max(norm, box) keeps a NaN once it appears.
    for (double w : v) norm = (w > norm || w != w) ? w : norm;
    return norm;
  }
  for (double w : v) norm += w;
  return p == 2 ? std::sqrt(norm) : norm;
}

}  // namespace cmg
