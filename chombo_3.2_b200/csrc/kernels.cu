// Device kernels of the AMR multigrid V-cycle.  Each kernel states the
// reference operation (ChF kernel or C++ routine, paths relative to the
// Chombo lib/src tree) whose arithmetic it reproduces term for term, so the
// FP64 build (compiled with --fmad=false) rounds exactly like the reference.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <stdexcept>

#include <cooperative_groups.h>

#include "kernels.H"
#include "synthdev.H"
#include "plan.H"
#include "synthetic.H"

namespace cg = cooperative_groups;

namespace cmg {

namespace {

inline void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "cmg: %s: %s", what, cudaGetErrorString(e));
    throw std::runtime_error(buf);
  }
}
std::atomic<long long> g_launches{0};
#define CMG_LAUNCHED(name) (g_launches.fetch_add(1, std::memory_order_relaxed), check(cudaGetLastError(), name))

// Cell q of box b in x-fastest order.
__device__ __forceinline__ bool allCell(const BoxDesc& b, int q, int& i, int& j, int& k) {
  int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
  if (q >= nx * ny * nz) return false;
  const int r = fastDiv(q, nx, b.mNx);
  const int kk = fastDiv(r, ny, b.mNy);
  i = b.lo[0] + (q - r * nx);
  j = b.lo[1] + (r - kk * ny);
  k = b.lo[2] + kk;
  return true;
}

// q-th cell of colour `color` (cells with i+j+k = color mod 2), the cells the
// GSRB kernels visit for redBlack = color (AMRPoissonOpF.ChF:151-158).
__device__ __forceinline__ bool colorCell(const BoxDesc& b, int q, int color, int& i, int& j, int& k) {
  int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
  int half = (nx + 1) / 2;
  const int r = fastDiv(q, half, b.mHalf);
  if (r >= ny * nz) return false;
  const int kk = fastDiv(r, ny, b.mNy);
  j = b.lo[1] + (r - kk * ny);
  k = b.lo[2] + kk;
  const int par = (b.lo[0] + j + k + color) & 1;
  i = b.lo[0] + par + 2 * (q - r * half);
  return i <= b.hi[0];
}

// ---------------------------------------------------------------- ghosts
// Exchange copies (BoxLayoutData local copy), homogeneous Dirichlet faces
// (BCFunc.cpp:25-32,294-354: ghost = 2*0 - near), homogeneous quadratic and
// linear coarse-fine ghosts (InterpF.ChF:435-494) and zeroing.
// Each thread takes GHOST_PER_THREAD ghost cells of its block's range; the
// task of cell g is found by binary search in the cumulative cell counts,
// between the tasks holding the first cells of this block and of the next
// (blockTask).  The cells' target and source indices are resolved first and
// their loads issued together.  par >= 0 fills only the ghost cells of colour
// par ((i+j+k) & 1 == par): a colour pass reads no ghost of its own colour,
// so the fill before it needs only the other one; then a task offers
// colourSlots() slots, stepping by two along its parity axis.
template <class T>
__global__ void __launch_bounds__(GHOST_THREADS) k_ghost(const GhostTaskDev* tasks, const int* start,
                                                         const int* blockTask, int ntask, int ncell, int par, T* f,
                                                         T c1, T c2, T flin) {
  const int b0 = blockTask[blockIdx.x], b1 = min(blockTask[blockIdx.x + 1], ntask - 1);
  int64_t dst[GHOST_PER_THREAD], s1[GHOST_PER_THREAD], s2[GHOST_PER_THREAD];
  int kind[GHOST_PER_THREAD];
#pragma unroll
  for (int u = 0; u < GHOST_PER_THREAD; ++u) {
    kind[u] = -1;
    dst[u] = s1[u] = s2[u] = 0;
    const int g0 = blockIdx.x * GHOST_PER_BLOCK + u * GHOST_THREADS + threadIdx.x;
    if (g0 >= ncell) continue;
    int lo = b0, hi = b1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= g0)
        lo = mid;
      else
        hi = mid - 1;
    }
    const GhostTaskDev& t = tasks[lo];
    int q = g0 - start[lo], c[3];
    if (par < 0) {
      const int nx = t.hi[0] - t.lo[0] + 1, ny = t.hi[1] - t.lo[1] + 1;
      c[0] = t.lo[0] + q % nx;
      int r = q / nx;
      c[1] = t.lo[1] + r % ny;
      c[2] = t.lo[2] + r / ny;
    } else {
      const int a = t.ax, d1 = a == 0 ? 1 : 0, d2 = a == 2 ? 1 : 2;
      const int ha = (t.hi[a] - t.lo[a] + 2) >> 1, n1 = t.hi[d1] - t.lo[d1] + 1;
      int r = q / ha;
      c[d1] = t.lo[d1] + r % n1;
      c[d2] = t.lo[d2] + r / n1;
      c[a] = t.lo[a] + ((par - t.lo[a] - c[d1] - c[d2]) & 1) + 2 * (q % ha);
      if (c[a] > t.hi[a]) continue;
    }
    kind[u] = t.kind;
    dst[u] = cellIndex(t.dst, c[0], c[1], c[2]);
    if (t.kind == G_COPY) {
      s1[u] = cellIndex(t.src, c[0] - t.shift[0], c[1] - t.shift[1], c[2] - t.shift[2]);
    } else if (t.kind != G_ZERO) {
      int e[3] = {0, 0, 0};
      e[t.dir] = -t.side;  // one cell inward
      s1[u] = cellIndex(t.dst, c[0] + e[0], c[1] + e[1], c[2] + e[2]);
      s2[u] = t.kind == G_CFQUAD ? cellIndex(t.dst, c[0] + 2 * e[0], c[1] + 2 * e[1], c[2] + 2 * e[2]) : s1[u];
    }
  }
  T v1[GHOST_PER_THREAD], v2[GHOST_PER_THREAD];
#pragma unroll
  for (int u = 0; u < GHOST_PER_THREAD; ++u) {
    if (kind[u] > 0 && kind[u] != G_ZERO) v2[u] = f[s2[u]];
    if (kind[u] >= 0 && kind[u] != G_ZERO) v1[u] = f[s1[u]];
  }
#pragma unroll
  for (int u = 0; u < GHOST_PER_THREAD; ++u) {
    const int k = kind[u];
    if (k < 0) continue;
    T out;
    if (k == G_COPY) {
      out = v1[u];
    } else if (k == G_ZERO) {
      out = T(0);
    } else if (k == G_BC) {
      T zero = T(0);
      out = T(2) * zero - v1[u];
    } else if (k == G_NEU) {
      out = v1[u];
    } else if (k == G_CFLIN) {
      out = flin * v1[u];
    } else {
      out = c1 * v1[u] + c2 * v2[u];
    }
    f[dst[u]] = out;
  }
}

// Ghost fill from the flat per-cell lists: entries [a0, a1) then [b0, b1),
// U per thread (GHOST_THREADS apart, so each batch of loads is coalesced),
// no table walk between a thread and its data.  A fill's sources are valid
// cells and its destinations ghost cells, so all loads of a thread are
// issued before its stores: the list and source latencies of its U entries
// overlap instead of adding up.
template <class T, int U>
__global__ void __launch_bounds__(GHOST_THREADS) k_ghostcells(const GhostCell* __restrict__ e, int a0, int a1,
                                                              int b0, int b1, T* f, T c1, T c2, T flin) {
  const int na = a1 - a0, n = na + (b1 - b0);
  const int base = blockIdx.x * (GHOST_THREADS * U) + threadIdx.x;
  GhostCell g[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int q = base + u * GHOST_THREADS;
    g[u] = q < n ? e[q < na ? a0 + q : b0 + (q - na)] : GhostCell{-1, 0, -1};
  }
  T v1[U], v2[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    v1[u] = g[u].dst >= 0 ? f[g[u].s1] : T(0);
    v2[u] = g[u].dst >= 0 && g[u].s2 >= 0 ? f[g[u].s2] : T(0);
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (g[u].dst < 0) continue;
    T out;
    if (g[u].s2 == -1) {
      out = v1[u];
    } else if (g[u].s2 == -2) {
      T zero = T(0);
      out = T(2) * zero - v1[u];
    } else if (g[u].s2 == -3) {
      out = flin * v1[u];
    } else {
      out = c1 * v1[u] + c2 * v2[u];
    }
    f[g[u].dst] = out;
  }
}

// ---------------------------------------------------------------- stencils
// Sum of the six neighbours in the ChF order (+x, -x, +y, -y, +z, -z).
template <class T>
__device__ __forceinline__ T nbrSum(const T* p, const Stencil& st) {
  return p[st.xp] + p[st.xm] + p[st.yp] + p[st.ym] + p[st.zp] + p[st.zm];
}

// Variable-coefficient divergence term of VCAMRPoissonOpF.ChF:93-111 (the
// face above the cell in direction d is stored at the neighbour's index).
template <class T>
__device__ __forceinline__ T vcDiv(const T* p, const T* b0, const T* b1, const T* b2, const Stencil& st) {
  T pc = p[st.c];
  return b0[st.xp] * (p[st.xp] - pc) - b0[st.c] * (pc - p[st.xm]) + b1[st.yp] * (p[st.yp] - pc) -
         b1[st.c] * (pc - p[st.ym]) + b2[st.zp] * (p[st.zp] - pc) - b2[st.c] * (pc - p[st.zm]);
}

struct Scal {
  double dxinv, lambda, alpha, beta;
  int laplacian;
};

// Value of the face ghost of box b beyond cell (i,j,k) in direction d on
// side s, from its fill rule (FaceRule); pc is the cell's current value.
struct GhostCoef {
  double c1, c2, flin;
};
template <class T>
__device__ __forceinline__ T ghostValue(const FaceRule* __restrict__ rules, const int* __restrict__ faceOff,
                                        const BoxDesc& bd, int b, int d, int s, int i, int j, int k, T pc,
                                        const T* phi, const GhostCoef& gc) {
  const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
  const int p[3] = {i, j, k};
  const FaceRule r = rules[faceOff[6 * b + 2 * d + (s > 0)] + (p[t0] - bd.lo[t0]) +
                           (bd.hi[t0] - bd.lo[t0] + 1) * (p[t1] - bd.lo[t1])];
  if (r.kind == FR_COPY || r.kind == FR_FAB) return phi[r.src];
  if (r.kind == FR_NEU) return pc;
  if (r.kind == FR_BC) {
    T zero = T(0);
    return T(2) * zero - pc;
  }
  if (r.kind == FR_CFLIN) return T(gc.flin) * pc;
  return T(gc.c1) * pc + T(gc.c2) * phi[r.src];
}

// Value of one ghost-fill entry (GhostCell) from the current field: the
// arithmetic of k_ghostcells.
template <class T>
__device__ __forceinline__ T ghostCellValue(const GhostCell& g, const T* f, const GhostCoef& gc) {
  const T v1 = f[g.s1];
  if (g.s2 == -1) return v1;
  if (g.s2 == -2) {
    T zero = T(0);
    return T(2) * zero - v1;
  }
  if (g.s2 == -3) return T(gc.flin) * v1;
  return T(gc.c1) * v1 + T(gc.c2) * f[g.s2];
}

// GSRBLAPLACIAN / GSRBHELMHOLTZ (AMRPoissonOpF.ChF:51-198) and
// GSRBHELMHOLTZVC3D (VCAMRPoissonOpF.ChF:57-125), one colour.  With PRE, the
// block first writes the face ghosts its own cells read (the chunk's entries
// of the fill that would precede the pass, pre[preStart[chunk] ..
// preStart[chunk + 1])).  Those ghosts belong to the other colour, so no other
// block writes their sources during the pass, and each is read only by the
// one valid cell next to it, updated by this block after the barrier: the
// values are the fill's.
template <class T, int VC, bool PRE>
__global__ void k_gsrb(const BoxDesc* boxes, const Chunk* chunks, T* phi, const T* rhs, int color, Scal sc,
                       const T* a, const T* b0, const T* b1, const T* b2, const T* lam,
                       const GhostCell* __restrict__ pre, const int* __restrict__ preStart, GhostCoef gc) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  if (PRE) {
    const int g1 = preStart[blockIdx.x + 1];
    for (int q = preStart[blockIdx.x] + threadIdx.x; q < g1; q += blockDim.x) {
      const GhostCell g = pre[q];
      phi[g.dst] = ghostCellValue(g, phi, gc);
    }
    __syncthreads();
  }
  int i, j, k;
  if (!colorCell(bd, ch.start + threadIdx.x, color, i, j, k)) return;
  const Stencil st = stencil(bd, i, j, k);
  const int64_t c = st.c;
  const T pc = phi[c];
  T v[6];
  v[0] = phi[st.xp];
  v[1] = phi[st.xm];
  v[2] = phi[st.yp];
  v[3] = phi[st.ym];
  v[4] = phi[st.zp];
  v[5] = phi[st.zm];
  const T dxinv = T(sc.dxinv);
  if (VC) {
    T div = b0[st.xp] * (v[0] - pc) - b0[c] * (pc - v[1]) + b1[st.yp] * (v[2] - pc) - b1[c] * (pc - v[3]) +
            b2[st.zp] * (v[4] - pc) - b2[c] * (pc - v[5]);
    T lofphi = T(sc.alpha) * a[c] * pc - T(sc.beta) * div * dxinv;
    phi[c] = pc - lam[c] * (lofphi - rhs[c]);
  } else if (sc.laplacian) {
    T lphi = (v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) * dxinv;
    phi[c] = T(sc.lambda) * (rhs[c] - lphi);
  } else {
    T lphi = ((v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) - T(2.0) * T(3) * pc) * dxinv;
    T helmop = T(sc.alpha) * pc + T(sc.beta) * lphi;
    phi[c] = pc + T(sc.lambda) * (helmop - rhs[c]);
  }
}

// One GSRB update (k_gsrb's arithmetic) from loaded values: v the six
// neighbours (+x, -x, +y, -y, +z, -z), f the face coefficients
// (b0[+x], b0[c], b1[+y], b1[c], b2[+z], b2[c]) of a VC operator.
template <class T, int VC>
__device__ __forceinline__ T gsrbValue(const Scal& sc, T pc, T rh, const T* v, T av, T lv, const T* f) {
  const T dxinv = T(sc.dxinv);
  if (VC) {
    T div = f[0] * (v[0] - pc) - f[1] * (pc - v[1]) + f[2] * (v[2] - pc) - f[3] * (pc - v[3]) + f[4] * (v[4] - pc) -
            f[5] * (pc - v[5]);
    T lofphi = T(sc.alpha) * av * pc - T(sc.beta) * div * dxinv;
    return pc - lv * (lofphi - rh);
  } else if (sc.laplacian) {
    T lphi = (v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) * dxinv;
    return T(sc.lambda) * (rh - lphi);
  } else {
    T lphi = ((v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) - T(2.0) * T(3) * pc) * dxinv;
    T helmop = T(sc.alpha) * pc + T(sc.beta) * lphi;
    return pc + T(sc.lambda) * (helmop - rh);
  }
}

// The one-colour pass of k_gsrb (ghosts filled before the pass) with two
// cells per thread: colour indices q and q + 1 of the chunk, which for an
// even number of colour cells per row are neighbours in one row (i and
// i + 2), sharing the enumeration, the index arithmetic and the x-neighbour
// between them (phi[oth + xo] is +x of the first and -x of the second).  A
// pair split across rows (odd rows) takes the second cell's own indices.
// All loads come before both stores (cells of one colour read only the other
// colour and themselves), so the two updates are those of k_gsrb.
template <class T, int VC>
__device__ __forceinline__ void gsrbOne(const BoxDesc& bd, int i, int j, int k, T* phi, const T* rhs, const Scal& sc,
                                        const T* a, const T* b0, const T* b1, const T* b2, const T* lam) {
  const Stencil s = stencil(bd, i, j, k);
  const T v[6] = {phi[s.xp], phi[s.xm], phi[s.yp], phi[s.ym], phi[s.zp], phi[s.zm]};
  T f[6], av = T(0), lv = T(0);
  if (VC) {
    av = a[s.c];
    lv = lam[s.c];
    f[0] = b0[s.xp];
    f[1] = b0[s.c];
    f[2] = b1[s.yp];
    f[3] = b1[s.c];
    f[4] = b2[s.zp];
    f[5] = b2[s.c];
  }
  phi[s.c] = gsrbValue<T, VC>(sc, phi[s.c], rhs[s.c], v, av, lv, f);
}

// The one-colour pass of k_gsrb (ghosts filled before the pass) with two
// cells per thread: colour indices q and q + 1 of the chunk, which for an
// even number of colour cells per row are neighbours in one row (i and
// i + 2), sharing the enumeration, the index arithmetic and the x-neighbour
// between them (phi[oth + xo] is +x of the first and -x of the second).  A
// pair split across rows (odd rows) updates its cells one by one.  All loads
// of a pair come before its stores (cells of one colour read only the other
// colour and themselves), so the updates are those of k_gsrb.
template <class T, int VC>
__global__ void __launch_bounds__(CHUNK / 2) k_gsrb_pair(const BoxDesc* boxes, const Chunk* chunks, T* phi,
                                                         const T* rhs, int color, Scal sc, const T* a, const T* b0,
                                                         const T* b1, const T* b2, const T* lam) {
  const Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  const int q = ch.start + 2 * threadIdx.x;
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1, nz = bd.hi[2] - bd.lo[2] + 1;
  const int half = (nx + 1) / 2;
  const int r = fastDiv(q, half, bd.mHalf);
  if (r >= ny * nz) return;
  const int kk = fastDiv(r, ny, bd.mNy);
  const int j = bd.lo[1] + (r - kk * ny), k = bd.lo[2] + kk;
  const int m = q - r * half;
  const int i = bd.lo[0] + ((bd.lo[0] + j + k + color) & 1) + 2 * m;
  if (m + 1 < half && i + 2 <= bd.hi[0]) {
    // both cells in this row
    const Stencil st = stencil(bd, i, j, k);
    const int c = st.c;
    const T pc0 = phi[c], pc1 = phi[c + 1];
    const T rh0 = rhs[c], rh1 = rhs[c + 1];
    const T xm = phi[st.xm], xc = phi[st.xp], xp = phi[st.xp + 1];
    const T v0[6] = {xc, xm, phi[st.yp], phi[st.ym], phi[st.zp], phi[st.zm]};
    const T v1[6] = {xp, xc, phi[st.yp + 1], phi[st.ym + 1], phi[st.zp + 1], phi[st.zm + 1]};
    T av0 = T(0), av1 = T(0), lv0 = T(0), lv1 = T(0), f0[6], f1[6];
    if (VC) {
      av0 = a[c];
      av1 = a[c + 1];
      lv0 = lam[c];
      lv1 = lam[c + 1];
      f0[0] = b0[st.xp];
      f0[1] = b0[c];
      f0[2] = b1[st.yp];
      f0[3] = b1[c];
      f0[4] = b2[st.zp];
      f0[5] = b2[c];
      f1[0] = b0[st.xp + 1];
      f1[1] = b0[c + 1];
      f1[2] = b1[st.yp + 1];
      f1[3] = b1[c + 1];
      f1[4] = b2[st.zp + 1];
      f1[5] = b2[c + 1];
    }
    const T n0 = gsrbValue<T, VC>(sc, pc0, rh0, v0, av0, lv0, f0);
    const T n1 = gsrbValue<T, VC>(sc, pc1, rh1, v1, av1, lv1, f1);
    phi[c] = n0;
    phi[c + 1] = n1;
    return;
  }
  if (i <= bd.hi[0]) gsrbOne<T, VC>(bd, i, j, k, phi, rhs, sc, a, b0, b1, b2, lam);
  int i1, j1, k1;
  if (colorCell(bd, q + 1, color, i1, j1, k1)) gsrbOne<T, VC>(bd, i1, j1, k1, phi, rhs, sc, a, b0, b1, b2, lam);
}

// n red-black sweeps of a small level in one launch: one block walks every
// cell of a colour (ghosts from their rules), synchronises, and goes on to
// the next colour and sweep -- the launches of 2n colour passes replaced by
// block barriers.  Same cell updates in the same colour order.
template <class T, int VC>
__global__ void __launch_bounds__(1024) k_relax_block(const BoxDesc* boxes, const Chunk* ch0, int n0,
                                                      const Chunk* ch1, int n1, T* phi, const T* rhs, Scal sc,
                                                      const T* a, const T* b0, const T* b1, const T* b2,
                                                      const T* lam, const FaceRule* __restrict__ rules,
                                                      const int* __restrict__ faceOff, GhostCoef gc, int nsweeps) {
  const T dxinv = T(sc.dxinv);
  for (int it = 0; it < nsweeps; ++it)
    for (int color = 0; color <= 1; ++color) {
      const Chunk* chunks = color ? ch1 : ch0;
      const int total = (color ? n1 : n0) * CHUNK;
      for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const Chunk ch = chunks[idx / CHUNK];
        const BoxDesc bd = boxes[ch.box];
        int i, j, k;
        if (!colorCell(bd, ch.start + idx % CHUNK, color, i, j, k)) continue;
        const Stencil st = stencil(bd, i, j, k);
        const int64_t c = st.c;
        const T pc = phi[c];
        const int b = ch.box;
        T v[6];
        v[0] = i == bd.hi[0] ? ghostValue(rules, faceOff, bd, b, 0, 1, i, j, k, pc, phi, gc) : phi[st.xp];
        v[1] = i == bd.lo[0] ? ghostValue(rules, faceOff, bd, b, 0, -1, i, j, k, pc, phi, gc) : phi[st.xm];
        v[2] = j == bd.hi[1] ? ghostValue(rules, faceOff, bd, b, 1, 1, i, j, k, pc, phi, gc) : phi[st.yp];
        v[3] = j == bd.lo[1] ? ghostValue(rules, faceOff, bd, b, 1, -1, i, j, k, pc, phi, gc) : phi[st.ym];
        v[4] = k == bd.hi[2] ? ghostValue(rules, faceOff, bd, b, 2, 1, i, j, k, pc, phi, gc) : phi[st.zp];
        v[5] = k == bd.lo[2] ? ghostValue(rules, faceOff, bd, b, 2, -1, i, j, k, pc, phi, gc) : phi[st.zm];
        if (VC) {
          T div = b0[st.xp] * (v[0] - pc) - b0[c] * (pc - v[1]) + b1[st.yp] * (v[2] - pc) - b1[c] * (pc - v[3]) +
                  b2[st.zp] * (v[4] - pc) - b2[c] * (pc - v[5]);
          T lofphi = T(sc.alpha) * a[c] * pc - T(sc.beta) * div * dxinv;
          phi[c] = pc - lam[c] * (lofphi - rhs[c]);
        } else if (sc.laplacian) {
          T lphi = (v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) * dxinv;
          phi[c] = T(sc.lambda) * (rhs[c] - lphi);
        } else {
          T lphi = ((v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) - T(2.0) * T(3) * pc) * dxinv;
          T helmop = T(sc.alpha) * pc + T(sc.beta) * lphi;
          phi[c] = pc + T(sc.lambda) * (helmop - rhs[c]);
        }
      }
      __syncthreads();
    }
}

// Neighbour value across a box face from its fill rule (the value the ghost
// fill before the colour pass would have written, as in ghostValue).
template <class T>
__device__ __forceinline__ T ruleValue(const FaceRule& r, T pc, const T* phi, const GhostCoef& gc) {
  if (r.kind == FR_COPY || r.kind == FR_FAB) return phi[r.src];
  if (r.kind == FR_NEU) return pc;
  if (r.kind == FR_BC) {
    T zero = T(0);
    return T(2) * zero - pc;
  }
  if (r.kind == FR_CFLIN) return T(gc.flin) * pc;
  return T(gc.c1) * pc + T(gc.c2) * phi[r.src];
}

// One cell of a red-black sweep with the neighbours beyond its box taken from
// the face rules: the arithmetic of k_gsrb (GSRBHELMHOLTZVC3D,
// GSRBLAPLACIAN, GSRBHELMHOLTZ).  With deferCopy, a cell with an exchange-copy
// face ghost is left alone (its source box may not be done yet).
template <class T, int VC>
__device__ __forceinline__ void gsrbCell(const BoxDesc& bd, int b, int i, int j, int k, T* phi, const T* rhs,
                                         const Scal& sc, const T* a, const T* b0, const T* b1, const T* b2,
                                         const T* lam, const FaceRule* __restrict__ rules,
                                         const int* __restrict__ faceOff, const GhostCoef& gc, bool deferCopy) {
  const Stencil st = stencil(bd, i, j, k);
  const int64_t c = st.c;
  const int p[3] = {i, j, k};
  const int nb[6] = {st.xp, st.xm, st.yp, st.ym, st.zp, st.zm};
  FaceRule fr[6];
  bool onFace[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int d = f >> 1, side = (f & 1) ? 0 : 1;  // +d then -d
    onFace[f] = side ? p[d] == bd.hi[d] : p[d] == bd.lo[d];
    if (onFace[f]) {
      const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
      fr[f] = rules[faceOff[6 * b + 2 * d + side] + (p[t0] - bd.lo[t0]) + (bd.hi[t0] - bd.lo[t0] + 1) * (p[t1] - bd.lo[t1])];
      if (deferCopy && fr[f].kind == FR_COPY) return;
    }
  }
  const T pc = phi[c];
  T v[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) v[f] = onFace[f] ? ruleValue(fr[f], pc, phi, gc) : phi[nb[f]];
  const T dxinv = T(sc.dxinv);
  if (VC) {
    T div = b0[st.xp] * (v[0] - pc) - b0[c] * (pc - v[1]) + b1[st.yp] * (v[2] - pc) - b1[c] * (pc - v[3]) +
            b2[st.zp] * (v[4] - pc) - b2[c] * (pc - v[5]);
    T lofphi = T(sc.alpha) * a[c] * pc - T(sc.beta) * div * dxinv;
    phi[c] = pc - lam[c] * (lofphi - rhs[c]);
  } else if (sc.laplacian) {
    T lphi = (v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) * dxinv;
    phi[c] = T(sc.lambda) * (rhs[c] - lphi);
  } else {
    T lphi = ((v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) - T(2.0) * T(3) * pc) * dxinv;
    T helmop = T(sc.alpha) * pc + T(sc.beta) * lphi;
    phi[c] = pc + T(sc.lambda) * (helmop - rhs[c]);
  }
}

// The fused sweep (gsrbSweepFused), first launch: one block per box marching
// through its z slabs.  Step s updates the colour-0 cells of slab s, then
// (after a barrier) the colour-1 cells of slab s - 1 except those with an
// exchange-copy face ghost.  Every read is the value the reference's two
// passes read: a colour-0 cell sees colour-1 neighbours not yet updated (slab
// s - 1 is updated after the barrier, slabs s and s + 1 in later steps, the
// other boxes' face cells only in the second launch), and a colour-1 cell sees
// the new colour-0 values of slabs s - 2 .. s of its own box; its coarse-fine
// and boundary ghosts use only its own box.  Part 2 of a step and part 1 of
// the next touch disjoint cells (slab s - 1 colour 1 against slab s + 1 colour
// 0 and its colour-1 neighbours in slabs s .. s + 2), so one barrier per step
// suffices.  The face coefficients and phi of a slab are read by both colours
// one step apart, from cache.
template <class T, int VC>
__global__ void __launch_bounds__(256) k_gsrb_march(const BoxDesc* boxes, T* phi, const T* rhs, Scal sc,
                                                    const T* a, const T* b0, const T* b1, const T* b2,
                                                    const T* lam, const FaceRule* __restrict__ rules,
                                                    const int* __restrict__ faceOff, GhostCoef gc) {
  const int b = blockIdx.x;
  const BoxDesc bd = boxes[b];
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1, nz = bd.hi[2] - bd.lo[2] + 1;
  const int half = (nx + 1) / 2;
  const int perSlab = half * ny;
  for (int s = 0; s <= nz; ++s) {
    if (s < nz) {
      const int k = bd.lo[2] + s;
      for (int q = threadIdx.x; q < perSlab; q += blockDim.x) {
        const int r = fastDiv(q, half, bd.mHalf);
        const int j = bd.lo[1] + r;
        const int i = bd.lo[0] + ((bd.lo[0] + j + k) & 1) + 2 * (q - r * half);
        if (i <= bd.hi[0]) gsrbCell<T, VC>(bd, b, i, j, k, phi, rhs, sc, a, b0, b1, b2, lam, rules, faceOff, gc, false);
      }
    }
    __syncthreads();
    if (s > 0) {
      const int k = bd.lo[2] + s - 1;
      for (int q = threadIdx.x; q < perSlab; q += blockDim.x) {
        const int r = fastDiv(q, half, bd.mHalf);
        const int j = bd.lo[1] + r;
        const int i = bd.lo[0] + ((bd.lo[0] + j + k + 1) & 1) + 2 * (q - r * half);
        if (i <= bd.hi[0]) gsrbCell<T, VC>(bd, b, i, j, k, phi, rhs, sc, a, b0, b1, b2, lam, rules, faceOff, gc, true);
      }
    }
  }
}

// The fused sweep, second launch: the colour-1 cells with an exchange-copy
// face ghost, now that every box has its new colour-0 values.
template <class T, int VC>
__global__ void __launch_bounds__(256) k_gsrb_deferred(const BoxDesc* boxes, const DeferredCell* cells, int n,
                                                       T* phi, const T* rhs, Scal sc, const T* a, const T* b0,
                                                       const T* b1, const T* b2, const T* lam,
                                                       const FaceRule* __restrict__ rules,
                                                       const int* __restrict__ faceOff, GhostCoef gc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const DeferredCell dc = cells[t];
  const BoxDesc bd = boxes[dc.box];
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1;
  const int r = fastDiv(dc.q, nx, bd.mNx);
  const int kk = fastDiv(r, ny, bd.mNy);
  gsrbCell<T, VC>(bd, dc.box, bd.lo[0] + (dc.q - r * nx), bd.lo[1] + (r - kk * ny), bd.lo[2] + kk, phi, rhs, sc, a,
                  b0, b1, b2, lam, rules, faceOff, gc, false);
}

// OPERATORLAPRES / OPERATORLAP (AMRPoissonOpF.ChF:287-377) and
// VCCOMPUTERES3D / VCCOMPUTEOP3D (VCAMRPoissonOpF.ChF:148-312) value of one
// cell from loaded values (v and f as in gsrbValue).  MODE 0: r = rhs - L(phi)
// (residual form), MODE 1: r = L(phi).
template <class T, int VC, int MODE>
__device__ __forceinline__ T opValue(const Scal& sc, T pc, T rh, const T* v, T av, const T* f) {
  const T dxinv = T(sc.dxinv);
  if (VC) {
    T div = f[0] * (v[0] - pc) - f[1] * (pc - v[1]) + f[2] * (v[2] - pc) - f[3] * (pc - v[3]) + f[4] * (v[4] - pc) -
            f[5] * (pc - v[5]);
    T lofphi = T(sc.alpha) * av * pc - T(sc.beta) * div * dxinv;
    return MODE == 0 ? rh - lofphi : lofphi;
  } else {
    T lap = ((v[0] + v[1] + v[2] + v[3] + v[4] + v[5]) - T(6) * pc) * dxinv;
    return MODE == 0 ? -(T(sc.alpha) * pc) - T(sc.beta) * lap + rh : T(sc.alpha) * pc + T(sc.beta) * lap;
  }
}

template <class T, int VC, int MODE>
__device__ __forceinline__ void opOne(const BoxDesc& bd, int i, int j, int k, T* r, const T* phi, const T* rhs,
                                      const Scal& sc, const T* a, const T* b0, const T* b1, const T* b2) {
  const Stencil s = stencil(bd, i, j, k);
  const T v[6] = {phi[s.xp], phi[s.xm], phi[s.yp], phi[s.ym], phi[s.zp], phi[s.zm]};
  T f[6], av = T(0);
  if (VC) {
    av = a[s.c];
    f[0] = b0[s.xp];
    f[1] = b0[s.c];
    f[2] = b1[s.yp];
    f[3] = b1[s.c];
    f[4] = b2[s.zp];
    f[5] = b2[s.c];
  }
  r[s.c] = opValue<T, VC, MODE>(sc, phi[s.c], MODE == 0 ? rhs[s.c] : T(0), v, av, f);
}

// The operator / residual over both colours with two same-row cells per
// thread (as k_gsrb_pair): threads 0-127 take the colour-0 cells of one
// colour chunk, threads 128-255 the colour-1 cells of the chunk with the same
// boundaries, so a block reads both colour halves of the same slots and each
// half finds its neighbours in the other's lines.
template <class T, int VC, int MODE>
__global__ void __launch_bounds__(CHUNK) k_op_pair(const BoxDesc* boxes, const Chunk* ch0, const Chunk* ch1, T* r,
                                                   const T* phi, const T* rhs, Scal sc, const T* a, const T* b0,
                                                   const T* b1, const T* b2) {
  const int color = threadIdx.x >= CHUNK / 2;
  const Chunk ch = (color ? ch1 : ch0)[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  const int q = ch.start + 2 * (threadIdx.x & (CHUNK / 2 - 1));
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1, nz = bd.hi[2] - bd.lo[2] + 1;
  const int half = (nx + 1) / 2;
  const int rr = fastDiv(q, half, bd.mHalf);
  if (rr >= ny * nz) return;
  const int kk = fastDiv(rr, ny, bd.mNy);
  const int j = bd.lo[1] + (rr - kk * ny), k = bd.lo[2] + kk;
  const int m = q - rr * half;
  const int i = bd.lo[0] + ((bd.lo[0] + j + k + color) & 1) + 2 * m;
  if (m + 1 < half && i + 2 <= bd.hi[0]) {
    const Stencil st = stencil(bd, i, j, k);
    const int c = st.c;
    const T pc0 = phi[c], pc1 = phi[c + 1];
    T rh0 = T(0), rh1 = T(0);
    if (MODE == 0) {
      rh0 = rhs[c];
      rh1 = rhs[c + 1];
    }
    const T xm = phi[st.xm], xc = phi[st.xp], xp = phi[st.xp + 1];
    const T v0[6] = {xc, xm, phi[st.yp], phi[st.ym], phi[st.zp], phi[st.zm]};
    const T v1[6] = {xp, xc, phi[st.yp + 1], phi[st.ym + 1], phi[st.zp + 1], phi[st.zm + 1]};
    T av0 = T(0), av1 = T(0), f0[6], f1[6];
    if (VC) {
      av0 = a[c];
      av1 = a[c + 1];
      f0[0] = b0[st.xp];
      f0[1] = b0[c];
      f0[2] = b1[st.yp];
      f0[3] = b1[c];
      f0[4] = b2[st.zp];
      f0[5] = b2[c];
      f1[0] = b0[st.xp + 1];
      f1[1] = b0[c + 1];
      f1[2] = b1[st.yp + 1];
      f1[3] = b1[c + 1];
      f1[4] = b2[st.zp + 1];
      f1[5] = b2[c + 1];
    }
    r[c] = opValue<T, VC, MODE>(sc, pc0, rh0, v0, av0, f0);
    r[c + 1] = opValue<T, VC, MODE>(sc, pc1, rh1, v1, av1, f1);
    return;
  }
  if (i <= bd.hi[0]) opOne<T, VC, MODE>(bd, i, j, k, r, phi, rhs, sc, a, b0, b1, b2);
  int i1, j1, k1;
  if (colorCell(bd, q + 1, color, i1, j1, k1)) opOne<T, VC, MODE>(bd, i1, j1, k1, r, phi, rhs, sc, a, b0, b1, b2);
}

template <class T>
__global__ void k_negadd(const BoxDesc* boxes, const Chunk* chunks, T* r, const T* lofphi, const T* rhs) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  int i, j, k;
  if (!allCell(bd, ch.start + threadIdx.x, i, j, k)) return;
  int64_t c = cellIndex(bd, i, j, k);
  r[c] = lofphi[c] * T(-1) + rhs[c] * T(1);
}

template <class T, class X>
__global__ void k_incr(const BoxDesc* boxes, const Chunk* chunks, T* lhs, const X* x, T scale) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  int i, j, k;
  if (!allCell(bd, ch.start + threadIdx.x, i, j, k)) return;
  int64_t c = cellIndex(bd, i, j, k);
  lhs[c] = lhs[c] + T(x[c]) * scale;
}

// lhs += x * scale and r = -lofphi + rhs over whole level arrays, ghost and
// padding slots included: the valid cells get exactly the reference's
// values, the ghost slots of these fields are rewritten by a ghost fill or
// coarse-fine interpolation before anything reads them, and one flat,
// perfectly coalesced loop beats walking the valid cells box by box.
template <class T, class X>
__global__ void k_incr_flat(T* lhs, const X* x, T scale, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    lhs[q] = lhs[q] + T(x[q]) * scale;
}
template <class T>
__global__ void k_negadd_flat(T* r, const T* lofphi, const T* rhs, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    r[q] = lofphi[q] * T(-1) + rhs[q] * T(1);
}
inline int flatBlocks(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

// x *= s over a whole level array (LevelDataOps::scale -> FArrayBox::mult).
__global__ void k_scale_flat(double* x, double s, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    x[q] = x[q] * s;
}

// Per-box dot products in the reference's order: FArrayBox::dotProduct
// (BoxTools/FArrayBox.cpp:260-280) accumulates x*y over the valid box k, j, i
// with i fastest into one running sum.  One warp per box: the lanes load and
// multiply a chunk of DOT_CHUNK consecutive cells (the products round the same
// whatever computes them) into shared memory, then lane 0 adds the chunk in
// order, so the sum is the reference's bit for bit; the sum over boxes and
// levels is left to the caller (LevelDataOps::dotProduct,
// MultilevelLinearOp::dotProduct).
enum { DOT_CHUNK = 512, DOT_PER_LANE = DOT_CHUNK / 32 };
__global__ void __launch_bounds__(32) k_box_dot(const BoxDesc* boxes, const double* __restrict__ x,
                                                const double* __restrict__ y, double* out) {
  __shared__ double prod[2][DOT_CHUNK];
  const BoxDesc bd = boxes[blockIdx.x];
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1, nz = bd.hi[2] - bd.lo[2] + 1;
  const int n = nx * ny * nz;
  const int lane = threadIdx.x;
  double xr[DOT_PER_LANE], yr[DOT_PER_LANE];
  // Loads of one chunk into registers (issued, not waited for).
  auto issue = [&](int base) {
#pragma unroll
    for (int u = 0; u < DOT_PER_LANE; ++u) {
      const int q = base + lane + 32 * u;
      xr[u] = 0.0;
      yr[u] = 0.0;
      if (q < n) {
        const int i = bd.lo[0] + q % nx, j = bd.lo[1] + (q / nx) % ny, k = bd.lo[2] + q / (nx * ny);
        const int64_t c = cellIndex(bd, i, j, k);
        xr[u] = x[c];
        yr[u] = y[c];
      }
    }
  };
  auto store = [&](double* dst) {
#pragma unroll
    for (int u = 0; u < DOT_PER_LANE; ++u) dst[lane + 32 * u] = xr[u] * yr[u];
  };
  double s = 0.0;
  issue(0);
  store(prod[0]);
  __syncwarp();
  for (int base = 0, buf = 0; base < n; base += DOT_CHUNK, buf ^= 1) {
    // the next chunk's loads are in flight while lane 0 adds this one
    const bool more = base + DOT_CHUNK < n;
    if (more) issue(base + DOT_CHUNK);
    if (lane == 0) {
      const int m = min(DOT_CHUNK, n - base);
      const double* p = prod[buf];
      for (int u = 0; u < m; ++u) s += p[u];
    }
    __syncwarp();
    if (more) store(prod[buf ^ 1]);
    __syncwarp();
  }
  if (lane == 0) out[blockIdx.x] = s;
}

// dst = src over whole arrays (ghosts included), converting the type.
template <class D, class S>
__global__ void k_convert(D* dst, const S* src, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    dst[q] = D(src[q]);
}

__device__ __forceinline__ void atomicMaxPos(double* addr, double v) {
  // v >= 0 or a NaN without sign: the IEEE bit pattern of a non-negative
  // double orders like an unsigned integer, so an integer max is a floating
  // max, and such a NaN (exponent all ones, mantissa non-zero) is above
  // every number, infinity included: a NaN anywhere wins.
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// max(a, b) that keeps a NaN from either side (fmax drops it).
__device__ __forceinline__ double nanMax(double a, double b) { return (b > a || b != b) ? b : a; }

template <class T>
__global__ void k_maxnorm(const BoxDesc* boxes, const Chunk* chunks, int nchunks, const T* f, double* out) {
  // Blocks stride over the chunks (one chunk each when the grid covers
  // them), so a large level sends one atomic per block, not per chunk.
  // Up to four chunks per step, their table loads and values issued
  // together (the max does not depend on the order).
  double v = 0.0;
  for (int c0 = blockIdx.x; c0 < nchunks; c0 += 4 * gridDim.x) {
    int64_t at[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      at[u] = -1;
      const int cix = c0 + u * gridDim.x;
      if (cix >= nchunks) continue;
      const Chunk ch = chunks[cix];
      const BoxDesc bd = boxes[ch.box];
      int i, j, k;
      if (allCell(bd, ch.start + threadIdx.x, i, j, k)) at[u] = cellIndex(bd, i, j, k);
    }
    double x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) x[u] = at[u] >= 0 ? fabs((double)f[at[u]]) : 0.0;
#pragma unroll
    for (int u = 0; u < 4; ++u) v = nanMax(v, x[u]);
  }
  for (int o = 16; o > 0; o >>= 1) v = nanMax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ double red[CHUNK / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < CHUNK / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = nanMax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) atomicMaxPos(out, fabs(v));
  }
}

// The max-norm of a forest level, one chunk per block, folded into the
// norm of the chunk's hierarchy.
template <class T>
__global__ void k_maxnorm_hier(const BoxDesc* boxes, const Chunk* chunks, const int* boxHier, const T* f,
                               double* out) {
  const Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  double v = 0.0;
  int i, j, k;
  if (allCell(bd, ch.start + threadIdx.x, i, j, k)) v = fabs((double)f[cellIndex(bd, i, j, k)]);
  for (int o = 16; o > 0; o >>= 1) v = nanMax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ double red[CHUNK / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < CHUNK / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = nanMax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) atomicMaxPos(out + boxHier[ch.box], fabs(v));
  }
}

// lhs += x over hierarchy blockIdx.y's element range of a forest level, if
// that hierarchy is still iterating (k_incr_flat's arithmetic).
template <class T, class X>
__global__ void k_incr_active(T* lhs, const X* x, const int64_t* hierStart, const int* active) {
  const int h = blockIdx.y;
  if (!active[h]) return;
  const int64_t a = hierStart[h], b = hierStart[h + 1];
  for (int64_t q = a + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < b; q += (int64_t)gridDim.x * blockDim.x)
    lhs[q] = lhs[q] + T(x[q]) * T(1.0);
}

// RESTRICTRES / RESTRICTRESVC3D (AMRPoissonOpF.ChF:394-438,
// VCAMRPoissonOpF.ChF:337-413): res_c accumulates (rhs - L phi)/8 over its 8
// fine cells in fine k-j-i order, starting from zero.
template <class T, int VC>
__global__ void k_restrictmg(const BoxDesc* fboxes, const BoxDesc* cboxes, const Chunk* chunks, T* resC,
                             const T* phi, const T* rhs, Scal sc, const T* a, const T* b0, const T* b1,
                             const T* b2) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc cb = cboxes[ch.box];
  int I, J, K;
  if (!allCell(cb, ch.start + threadIdx.x, I, J, K)) return;
  const BoxDesc fb = fboxes[ch.box];
  const T dxinv = T(sc.dxinv);
  const T denom = T(8);
  T acc = T(0);
  for (int kk = 0; kk < 2; ++kk)
    for (int jj = 0; jj < 2; ++jj)
      for (int ii = 0; ii < 2; ++ii) {
        const Stencil st = stencil(fb, 2 * I + ii, 2 * J + jj, 2 * K + kk);
        const int64_t c = st.c;
        T pc = phi[c];
        T lofphi;
        if (VC)
          lofphi = T(sc.alpha) * a[c] * pc - T(sc.beta) * vcDiv(phi, b0, b1, b2, st) * dxinv;
        else
          lofphi = T(sc.alpha) * pc + T(sc.beta) * (nbrSum(phi, st) - pc * T(2) * T(3)) * dxinv;
        acc = acc + (rhs[c] - lofphi) / denom;
      }
  resC[cellIndex(cb, I, J, K)] = acc;
}

// PROLONG (AMRPoissonOpF.ChF:453-478): phi += coarse(i/2), same box index.
template <class T>
__global__ void k_prolongmg(const BoxDesc* fboxes, const BoxDesc* cboxes, const Chunk* chunks, T* phi,
                            const T* corrC) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc fb = fboxes[ch.box];
  int i, j, k;
  if (!allCell(fb, ch.start + threadIdx.x, i, j, k)) return;
  int64_t c = cellIndex(fb, i, j, k);
  phi[c] = phi[c] + corrC[cellIndex(cboxes[ch.box], i >> 1, j >> 1, k >> 1)];
}

// AVERAGE with refRatio 2 (AverageF.ChF:36-55) written straight into the
// coarse level through the coarsened-fine -> coarse copy items.
template <class T>
__global__ void k_average(const BoxDesc* fboxes, const BoxDesc* cboxes, const CoarseFineItem* items,
                          const Chunk* chunks, T* coarse, const T* fine) {
  Chunk ch = chunks[blockIdx.x];
  const CoarseFineItem it = items[ch.box];
  int q = ch.start + threadIdx.x;
  int nx = it.hi[0] - it.lo[0] + 1, ny = it.hi[1] - it.lo[1] + 1, nz = it.hi[2] - it.lo[2] + 1;
  if (q >= nx * ny * nz) return;
  int I = it.lo[0] + q % nx, r = q / nx, J = it.lo[1] + r % ny, K = it.lo[2] + r / ny;
  const BoxDesc fb = fboxes[it.fbox];
  const int i = 2 * I, j = 2 * J, k = 2 * K;
  T sum = fine[cellIndex(fb, i, j, k)] + fine[cellIndex(fb, i + 1, j, k)] + fine[cellIndex(fb, i, j + 1, k)] +
          fine[cellIndex(fb, i + 1, j + 1, k)] + fine[cellIndex(fb, i, j, k + 1)] +
          fine[cellIndex(fb, i + 1, j, k + 1)] + fine[cellIndex(fb, i, j + 1, k + 1)] +
          fine[cellIndex(fb, i + 1, j + 1, k + 1)];
  coarse[cellIndex(cboxes[it.cbox], I, J, K)] = T(0.125) * sum;
}

// AMRProlongS (AMRPoissonOp.cpp:959-990): fine += coarse(i/2).  One thread
// per coarse cell of an item (chunks over the items' coarse cells, x
// fastest) updates its eight fine cells: the coarse value is read once, the
// eight fine loads are independent, and for each of the eight child offsets
// a warp's threads touch consecutive slots of one colour half.
template <class T>
__global__ void k_prolongamr(const BoxDesc* fboxes, const BoxDesc* cboxes, const CoarseFineItem* items,
                             const Chunk* chunks, T* fine, const T* coarse) {
  Chunk ch = chunks[blockIdx.x];
  const CoarseFineItem it = items[ch.box];
  const int q = ch.start + threadIdx.x;
  const int nx = it.hi[0] - it.lo[0] + 1, ny = it.hi[1] - it.lo[1] + 1, nz = it.hi[2] - it.lo[2] + 1;
  if (q >= nx * ny * nz) return;
  const int r = q / nx, kk = r / ny;
  const int I = it.lo[0] + (q - r * nx), J = it.lo[1] + (r - kk * ny), K = it.lo[2] + kk;
  const BoxDesc fb = fboxes[it.fbox];
  const T c = coarse[cellIndex(cboxes[it.cbox], I, J, K)];
  int64_t f[8];
  T v[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) f[n] = cellIndex(fb, 2 * I + (n & 1), 2 * J + ((n >> 1) & 1), 2 * K + (n >> 2));
#pragma unroll
  for (int n = 0; n < 8; ++n) v[n] = fine[f[n]];
#pragma unroll
  for (int n = 0; n < 8; ++n) fine[f[n]] = v[n] + c;
}

// lhs = lhs + x * 1 (k_incr_flat's arithmetic), then x = the new lhs: the
// increment followed by a copy back, in one pass.
template <class T>
__global__ void k_incr_copy_flat(T* lhs, T* x, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const T v = lhs[q] + x[q] * T(1.0);
    lhs[q] = v;
    x[q] = v;
  }
}

// lhs = lhs + x * 1, then x = 0: the increment followed by zeroing x.
template <class T>
__global__ void k_incr_zero_flat(T* lhs, T* x, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    lhs[q] = lhs[q] + x[q] * T(1.0);
    x[q] = T(0);
  }
}

// QuadCFStencil derivatives (AMRTools/QuadCFStencil.cpp:33-260).
template <class T>
__device__ __forceinline__ T cfFirst(const CFDeriv& d, const double* w, const int64_t* off, const T* pc, T dxc) {
  if (d.kind == 1) return (pc[off[d.start + 1]] - pc[off[d.start]]) / (T(2.0) * dxc);
  if (d.kind == 0) return T(0);
  T v = T(0);
  for (int n = 0; n < d.n; ++n) v += T(w[d.start + n]) * pc[off[d.start + n]];
  return v / dxc;
}
template <class T>
__device__ __forceinline__ T cfSecond(const CFDeriv& d, const double* w, const int64_t* off, const T* pc, T dxc) {
  if (d.kind == 1)
    return (pc[off[d.start + 1]] + pc[off[d.start]] - T(2.0) * pc[off[d.start + 2]]) / (dxc * dxc);
  if (d.kind == 0) return T(0);
  T v = T(0);
  for (int n = 0; n < d.n; ++n) v += T(w[d.start + n]) * pc[off[d.start + n]];
  return v / (dxc * dxc);
}
template <class T>
__device__ __forceinline__ T cfMixed(const CFDeriv& d, const double* w, const int64_t* off, const T* pc, T dxc) {
  if (d.kind == 1) {
    const int64_t* o = off + d.start;  // ur, ul, lr, ll
    return (pc[o[0]] + pc[o[3]] - pc[o[2]] - pc[o[1]]) / (T(4.) * dxc * dxc);
  }
  if (d.kind == 0) return T(0);
  T v = T(0);
  for (int n = 0; n < d.n; ++n) v += T(w[d.start + n]) * pc[off[d.start + n]];
  return v / (dxc * dxc);
}

// QuadCFInterp::getPhiStar + interpOnIVS (AMRTools/QuadCFInterp.cpp:569-839),
// in two launches.  First, per coarse cell under a coarse-fine face: the
// tangential first and second derivatives, the mixed derivative and the
// coarse value (six values into tmp); every fine ghost over that coarse cell
// (four on a face) reads them instead of gathering the stencils again.
template <class T>
__global__ void k_cf_coarse(const CFCoarse* coarse, int n, const double* w, const int64_t* off, const T* phiC, T h,
                            T* tmp) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const CFCoarse cc = coarse[t];
  const T dxc = T(2) * h;
  T* o = tmp + 6 * (int64_t)t;
  o[0] = cfFirst(cc.d1[0], w, off, phiC, dxc);
  o[1] = cfSecond(cc.d2[0], w, off, phiC, dxc);
  o[2] = cfFirst(cc.d1[1], w, off, phiC, dxc);
  o[3] = cfSecond(cc.d2[1], w, off, phiC, dxc);
  o[4] = cfMixed(cc.mx, w, off, phiC, dxc);
  o[5] = phiC[cc.cc];
}

// Second, per fine ghost: phistar from the coarse Taylor expansion, then the
// quadratic through phistar and two fine cells, in the Fortran (packed face,
// QuadCFInterpF.ChF:9-48) or C++ (unpacked face) arithmetic.
template <class T>
__global__ void k_quadcf(const CFFine* fine, int n, const T* tmp, T* phiF, T h) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const CFFine e = fine[t];
  const T* c = tmp + 6 * (int64_t)e.coarse;
  const T s1 = c[0], c1 = c[1], s2 = c[2], c2 = c[3], mx = c[4];
  const T x1 = T(e.x1), x2 = T(e.x2);
  T update1 = x1 * s1 + T(0.5) * x1 * x1 * c1;
  T update2 = x2 * s2 + T(0.5) * x2 * x2 * c2;
  T update3 = x1 * x2 * mx;
  T ps = c[5] + update1 + update2 + update3;
  T pa = phiF[e.pa], pb = phiF[e.pb];
  T r;
  if (e.packed) {
    T frac = T(2.0) / (h * h);
    T denom = T(2 * 2 + 4 * 2 + 3);
    T mult = frac / denom;
    T invh = T(1.0) / h;
    T x = T(2.0) * h;
    T xsq = T(4.0) * h * h;
    T a = mult * (T(2.0) * ps + T(2 + 1) * pa - T(2 + 3) * pb);
    T b = (pb - pa) * invh - a * h;
    r = xsq * a + b * x + pa;
  } else {
    T a = (T(2.) / h / h) * (T(2.) * ps + pa * (T(2) + T(1.0)) - pb * (T(2) + T(3.0))) / (T(2 * 2 + 4 * 2) + T(3.0));
    T b = (pb - pa) / h - a * h;
    T x = T(2.) * h;
    r = a * x * x + b * x + pa;
  }
  phiF[e.g] = r;
}

// Flux-register correction (AMRPoissonOp::reflux, VCAMRPoissonOp2::reflux
// and LevelFluxRegister incrementCoarse/incrementFine/reflux).
template <class T, int VC>
__global__ void k_reflux(const RefluxCell* cells, int n, const RefluxCoarseTerm* cterms, const RefluxFineGroup* fgroups,
                         T* lofphi, const T* phiC, const T* phiF, const T* bc0, const T* bc1, const T* bc2,
                         const T* bf0, const T* bf1, const T* bf2, T sc, T sf, T negs) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const RefluxCell rc = cells[t];
  const T* bc[3] = {bc0, bc1, bc2};
  const T* bf[3] = {bf0, bf1, bf2};
  T u = lofphi[rc.c];
  T coar = T(0);
  for (int m = 0; m < rc.nco; ++m) {
    const RefluxCoarseTerm ct = cterms[rc.start + m];
    T flux;
    if (VC)
      flux = -bc[ct.dir][ct.bface] * ((phiC[ct.hi] - phiC[ct.lo]) * sc);
    else
      flux = (phiC[ct.hi] - phiC[ct.lo]) * sc;
    coar = coar + flux * T(ct.sgn);
  }
  u = u + coar * negs;
  for (int m = 0; m < rc.nfi; ++m) {
    const RefluxFineGroup& g = fgroups[rc.fstart + m];
    T reg = T(0);
    for (int q = 0; q < 4; ++q) {
      T ff;
      if (VC)
        ff = -bf[g.dir][g.bface[q]] * ((phiF[g.hi[q]] - phiF[g.lo[q]]) * sf);
      else
        ff = (phiF[g.hi[q]] - phiF[g.lo[q]]) * sf;
      reg = reg + T(g.scale) * ff;
    }
    u = u + reg * negs;
  }
  lofphi[rc.c] = u;
}

// ---------------------------------------------------------------- bottom
// BiCGStabSolver<T>::solve (AMRElliptic/BiCGStabSolver.H:199-515) and
// RelaxSolver<T>::solve (RelaxSolver.H:128-186) on the deepest multigrid
// level, every dot product and norm summed in the reference's order: per box
// in x-fastest order (FArrayBox::dotProduct, FArrayBox.cpp:260-280;
// FArrayBox::sumPow pencil order, FArrayBox.cpp:168-209), then box by box
// from zero.  The vectors live in the bottom level's compact slot space (its
// valid cells, BottomPlan).  A stencil read of a face ghost goes straight to
// the valid cell that the level's exchange or boundary condition copies
// there (nbv: the source slot, or -(slot + 1) for a homogeneous Dirichlet
// ghost, read as 0 - value the way the BC writes it).  A ghost is only read
// while its source is not written (a colour pass reads the other colour; an
// operator apply writes another vector), so the value read is the one an
// exchange just before the pass would have left there.
// Two ways to run: one thread block per hierarchy (BlkCtx: forests and
// small levels), or the whole grid of one cooperative launch for one
// hierarchy with a large bottom level (GridCtx), its phases separated by
// grid barriers and its sums folded by block 0 from shared memory.
struct BottomArgs {
  BottomWork W;
  const BoxDesc* boxes;
  Scal sc;
  int vc;
  double* phiFab;
  const double* rhsFab;
  double *phi, *rhs, *r, *rt, *e, *p, *pt, *st, *t, *v;
  double eps, reps, hang, small, mult;
  const double* metric;  // device scalar: the solve's initial residual norm
  int imax, numRestarts;
  BottomConfig cfg;
  const double* epsPer;  // per block (hierarchy) tolerance of a BiCGStab bottom, or null
};

constexpr int kBottomGridThreads = 256;
constexpr int kBottomStage = 2048;  // doubles per fold chunk staged in shared memory (grid)

// In-order fold of p[0..n): a sum from zero, or a NaN-keeping max from zero.
__device__ __forceinline__ double foldRun(double acc, const double* p, int n, bool mx) {
  if (mx) {
    for (int b = 0; b < n; ++b) acc = nanMax(acc, p[b]);
  } else {
    for (int b = 0; b < n; ++b) acc += p[b];
  }
  return acc;
}

struct BlkCtx {
  static constexpr bool kGrid = false;
  double* part;   // per-box partials (dynamic shared memory)
  double* part2;  // a second set, for two sums folded together
  double* scal;   // 8 rotating broadcast slots (shared)
  int k;
  __device__ int tid() const { return threadIdx.x; }
  __device__ int nthr() const { return blockDim.x; }
  __device__ void sync() const { __syncthreads(); }
  // Folds part[0..n) (and part2 when two) once every thread has written its
  // partials; every thread gets the results.  A broadcast slot is written
  // again only four folds later, after every thread has read it.
  __device__ void reduce(int n, bool two, bool mx, double& r1, double& r2) {
    __syncthreads();
    const int s = k;
    k = (k + 2) & 7;
    if (threadIdx.x == 0) scal[s] = foldRun(0.0, part, n, mx);
    if (two && threadIdx.x == 32) scal[s + 1] = foldRun(0.0, part2, n, mx);
    __syncthreads();
    r1 = scal[s];
    if (two) r2 = scal[s + 1];
  }
};

struct GridCtx {
  static constexpr bool kGrid = true;
  double* part;   // per-box partials (global)
  double* part2;
  double* scal;   // 8 rotating broadcast slots (global)
  double* stage;  // 2 x kBottomStage doubles of shared memory
  int k;
  __device__ int tid() const { return blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ int nthr() const { return gridDim.x * blockDim.x; }
  __device__ void sync() const { cg::this_grid().sync(); }
  __device__ void reduce(int n, bool two, bool mx, double& r1, double& r2) {
    cg::this_grid().sync();
    const int s = k;
    k = (k + 2) & 7;
    if (blockIdx.x == 0) {
      double a1 = 0.0, a2 = 0.0;
      for (int base = 0; base < n; base += kBottomStage) {
        const int m = min(kBottomStage, n - base);
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
          stage[i] = __ldcg(part + base + i);
          if (two) stage[kBottomStage + i] = __ldcg(part2 + base + i);
        }
        __syncthreads();
        if (threadIdx.x == 0) a1 = foldRun(a1, stage, m, mx);
        if (two && threadIdx.x == 32) a2 = foldRun(a2, stage + kBottomStage, m, mx);
        __syncthreads();
      }
      if (threadIdx.x == 0) scal[s] = a1;
      if (two && threadIdx.x == 32) scal[s + 1] = a2;
    }
    cg::this_grid().sync();
    r1 = __ldcg(scal + s);
    if (two) r2 = __ldcg(scal + s + 1);
  }
};

template <class C, class F>
__device__ __forceinline__ void bCells(C& c, int n, F fn) {
  for (int q = c.tid(); q < n; q += c.nthr()) fn(q);
  c.sync();
}

// A face neighbour's value: the slot itself, or 0 - the source of a
// homogeneous Dirichlet ghost.
__device__ __forceinline__ double gval(const double* f, int v) { return v >= 0 ? f[v] : 0.0 - f[-v - 1]; }

// The partial sum of box b: x.y in x-fastest order, or sumPow(2) of x.
__device__ double boxPartial(const BottomArgs& A, int b, const double* x, const double* y, bool pencil) {
  const BoxDesc bd = A.boxes[b];
  const int nx = bd.hi[0] - bd.lo[0] + 1, ny = bd.hi[1] - bd.lo[1] + 1, nz = bd.hi[2] - bd.lo[2] + 1;
  const int s0 = A.W.boxStart[b];
  double s = 0.0;
  if (!pencil) {
    for (int q = s0; q < s0 + nx * ny * nz; ++q) s += x[q] * y[q];
  } else {
    // sumPow(p=2): per-x accumulation over pencils, then across x.
    for (int i = 0; i < nx; ++i) {
      double acc = 0.0;
      bool first = true;
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
          double v = x[s0 + i + nx * (j + ny * k)];
          acc = first ? v * v : acc + v * v;
          first = false;
        }
      s = (i == 0) ? acc : s + acc;
    }
  }
  return s;
}

template <class C>
__device__ double bDot(C& c, const BottomArgs& A, const double* x, const double* y, bool pencil) {
  for (int b = c.tid(); b < A.W.nbox; b += c.nthr()) c.part[b] = boxPartial(A, b, x, y, pencil);
  double r, unused;
  c.reduce(A.W.nbox, false, false, r, unused);
  return r;
}

// x1.y1 and x2.y2, each in the reference's order, folded side by side.
template <class C>
__device__ void bDot2(C& c, const BottomArgs& A, const double* x1, const double* y1, const double* x2,
                      const double* y2, double& r1, double& r2) {
  for (int b = c.tid(); b < A.W.nbox; b += c.nthr()) {
    c.part[b] = boxPartial(A, b, x1, y1, false);
    c.part2[b] = boxPartial(A, b, x2, y2, false);
  }
  c.reduce(A.W.nbox, true, false, r1, r2);
}

// The norm of type A.cfg.normType: 2 the reference-ordered sqrt(sumPow),
// 0 the largest |x| (a max, so its order does not matter; NaN propagates).
template <class C>
__device__ double bNormType(C& c, const BottomArgs& A, const double* x) {
  if (A.cfg.normType == 2) return sqrt(bDot(c, A, x, x, true));
  double v = 0.0;
  for (int q = c.tid(); q < A.W.nv; q += c.nthr()) v = nanMax(v, fabs(x[q]));
  for (int o = 16; o > 0; o >>= 1) v = nanMax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) c.part[c.tid() >> 5] = v;
  double r, unused;
  c.reduce(c.nthr() >> 5, false, true, r, unused);
  return r;
}

// One colour of levelGSRB, face ghosts read from their sources.
template <class C>
__device__ void bGsrb(C& c, const BottomArgs& A, double* phi, const double* rhs, int color) {
  const BottomWork& W = A.W;
  const int* list = W.col[color];
  const double dxinv = A.sc.dxinv;
  for (int idx = c.tid(); idx < W.ncol[color]; idx += c.nthr()) {
    const int q = list[idx];
    const int* n = W.nbv + 6 * q;
    const double pxp = gval(phi, n[0]), pxm = gval(phi, n[1]), pyp = gval(phi, n[2]), pym = gval(phi, n[3]),
                 pzp = gval(phi, n[4]), pzm = gval(phi, n[5]);
    const double pc = phi[q];
    if (A.vc) {
      const int* o = W.nb + 6 * q;
      const double div = W.b[0][o[0]] * (pxp - pc) - W.b[0][q] * (pc - pxm) + W.b[1][o[2]] * (pyp - pc) -
                         W.b[1][q] * (pc - pym) + W.b[2][o[4]] * (pzp - pc) - W.b[2][q] * (pc - pzm);
      const double lofphi = A.sc.alpha * W.a[q] * pc - A.sc.beta * div * dxinv;
      phi[q] = pc - W.lam[q] * (lofphi - rhs[q]);
    } else if (A.sc.laplacian) {
      const double lphi = (pxp + pxm + pyp + pym + pzp + pzm) * dxinv;
      phi[q] = A.sc.lambda * (rhs[q] - lphi);
    } else {
      const double lphi = (pxp + pxm + pyp + pym + pzp + pzm - 2.0 * 3 * pc) * dxinv;
      const double helmop = A.sc.alpha * pc + A.sc.beta * lphi;
      phi[q] = pc + A.sc.lambda * (helmop - rhs[q]);
    }
  }
  c.sync();
}

template <class C>
__device__ void bRelax(C& c, const BottomArgs& A, double* phi, const double* rhs, int nit) {
  for (int it = 0; it < nit; ++it)
    for (int color = 0; color <= 1; ++color) bGsrb(c, A, phi, rhs, color);
}

// residual (mode 0) or applyOp (mode 1) into every valid slot of r.
template <class C>
__device__ void bOp(C& c, const BottomArgs& A, double* r, const double* phi, const double* rhs, int mode) {
  const double dxinv = A.sc.dxinv;
  const BottomWork& W = A.W;
  bCells(c, W.nv, [&](int q) {
    const int* n = W.nbv + 6 * q;
    const double pxp = gval(phi, n[0]), pxm = gval(phi, n[1]), pyp = gval(phi, n[2]), pym = gval(phi, n[3]),
                 pzp = gval(phi, n[4]), pzm = gval(phi, n[5]);
    const double pc = phi[q];
    if (A.vc) {
      const int* o = W.nb + 6 * q;
      const double div = W.b[0][o[0]] * (pxp - pc) - W.b[0][q] * (pc - pxm) + W.b[1][o[2]] * (pyp - pc) -
                         W.b[1][q] * (pc - pym) + W.b[2][o[4]] * (pzp - pc) - W.b[2][q] * (pc - pzm);
      const double lofphi = A.sc.alpha * W.a[q] * pc - A.sc.beta * div * dxinv;
      r[q] = mode == 0 ? rhs[q] - lofphi : lofphi;
    } else {
      const double lap = (pxp + pxm + pyp + pym + pzp + pzm - 6.0 * pc) * dxinv;
      r[q] = mode == 0 ? -(A.sc.alpha * pc) - A.sc.beta * lap + rhs[q] : A.sc.alpha * pc + A.sc.beta * lap;
    }
  });
}

template <class C>
__device__ void bPrecond(C& c, const BottomArgs& A, double* out, const double* in) {
  bCells(c, A.W.nv, [&](int q) { out[q] = A.vc ? in[q] * A.W.lam[q] : in[q] * A.mult; });
  bRelax(c, A, out, in, 2);
}

// RelaxSolver<T>::solve (AMRElliptic/RelaxSolver.H:128-186): repeated
// preconditioner corrections e = preCond(r), phi += e, until the residual
// norm falls below eps times the initial one, imax iterations or a hang.
template <class C>
__device__ void bRelaxSolve(C& c, const BottomArgs& A) {
  const BottomWork& W = A.W;
  bOp(c, A, A.r, A.phi, A.rhs, 0);
  double norm = bNormType(c, A, A.r);
  double minNorm = norm;
  int iter = 0;
  if (norm > 0.) {
    const double initialNorm = norm;
    while (iter < A.cfg.imax) {
      bPrecond(c, A, A.e, A.r);
      bCells(c, W.nv, [&](int q) { A.phi[q] = A.phi[q] + A.e[q] * 1.0; });
      bOp(c, A, A.r, A.phi, A.rhs, 0);
      norm = bNormType(c, A, A.r);
      iter++;
      if (norm < A.cfg.eps * initialNorm) break;
      if (norm < minNorm)
        minNorm = norm;
      else if (norm * A.cfg.hang > minNorm)
        break;
    }
  }
  if (c.tid() == 0) W.status[0] = 0, W.status[1] = iter;
}

// On the grid, boxes of at most this many cells have their element-wise
// updates and their partial sums done by one thread each, with no barrier in
// between (in one block a barrier costs less than the serialised updates).
constexpr int kBoxWiseCells = 64;

// r += v * sv and e += w * sw on every valid slot, then the norm of r (and,
// with rtr, the reference-ordered rt.r, folded beside it): the two sums a
// BiCGStab half step ends with.
template <class C>
__device__ double bUpdateNorm(C& c, const BottomArgs& A, const double* v, double sv, const double* w, double sw,
                              double* rtr) {
  const BottomWork& W = A.W;
  if (C::kGrid && A.cfg.normType == 2 && W.maxBoxCells <= kBoxWiseCells) {
    for (int b = c.tid(); b < W.nbox; b += c.nthr()) {
      for (int q = W.boxStart[b]; q < W.boxStart[b + 1]; ++q) {
        A.r[q] = A.r[q] + v[q] * sv;
        A.e[q] = A.e[q] + w[q] * sw;
      }
      c.part[b] = boxPartial(A, b, A.r, A.r, true);
      if (rtr) c.part2[b] = boxPartial(A, b, A.rt, A.r, false);
    }
    double n2, d = 0.0;
    c.reduce(W.nbox, rtr != nullptr, false, n2, d);
    if (rtr) *rtr = d;
    return sqrt(n2);
  }
  bCells(c, W.nv, [&](int q) {
    A.r[q] = A.r[q] + v[q] * sv;
    A.e[q] = A.e[q] + w[q] * sw;
  });
  const double n = bNormType(c, A, A.r);
  if (rtr) *rtr = bDot(c, A, A.rt, A.r, false);
  return n;
}

// p from r (init) or p = (p beta + v (-beta omega)) + r, then the
// preconditioner pt = preCond(p): the two share their first pass.
template <class C>
__device__ void bDirection(C& c, const BottomArgs& A, bool init, double b1, double bo) {
  const BottomWork& W = A.W;
  bCells(c, W.nv, [&](int q) {
    double x;
    if (init) {
      x = A.r[q];
    } else {
      x = A.p[q] * b1;
      x = x + A.v[q] * bo;
      x = x + A.r[q] * 1.0;
    }
    A.p[q] = x;
    A.pt[q] = A.vc ? x * W.lam[q] : x * A.mult;
  });
  bRelax(c, A, A.pt, A.p, 2);
}

template <class C>
__device__ void bBicgstab(C& c, const BottomArgs& A) {
  const BottomWork& W = A.W;
  const int nv = W.nv;
  auto zeroV = [&](double* x) { bCells(c, nv, [&](int q) { x[q] = 0.0; }); };
  auto incrV = [&](double* y, const double* x, double sc) { bCells(c, nv, [&](int q) { y[q] = y[q] + x[q] * sc; }); };
  // rt = r, e = 0 in one pass
  auto restartVectors = [&]() {
    bCells(c, nv, [&](int q) {
      A.rt[q] = A.r[q];
      A.e[q] = 0.0;
    });
  };
  bOp(c, A, A.r, A.phi, A.rhs, 0);
  restartVectors();
  int iter = 0, recount = 0, restarts = 0, status = 0;
  double rho[4] = {0, 0, 0, 0};
  double norm[2];
  norm[0] = bNormType(c, A, A.r);
  double initial_norm = norm[0];
  const double initial_residual = norm[0];
  norm[1] = norm[0];
  double alpha[2] = {0, 0}, beta[2] = {0, 0}, omega[2] = {0, 0};
  bool init = true;
  // rt.r of the current r when the last half step folded it beside its norm
  bool haveRho = false;
  double rhoNext = 0.0;
  const double metric = *A.metric;
  if (metric > 0) initial_norm = metric;
  while ((iter < A.imax && norm[0] > A.eps * norm[1]) && (norm[1] > 0)) {
    iter++;
    norm[1] = norm[0];
    alpha[1] = alpha[0];
    beta[1] = beta[0];
    omega[1] = omega[0];
    rho[3] = rho[2];
    rho[2] = rho[1];
    rho[1] = haveRho ? rhoNext : bDot(c, A, A.rt, A.r, false);
    haveRho = false;
    if (rho[1] == 0.0) {
      incrV(A.phi, A.e, 1.0);
      if (c.tid() == 0) W.status[0] = 2, W.status[1] = iter;
      return;
    }
    double b1 = 0.0, bo = 0.0;
    if (!init) {
      beta[1] = (rho[1] / rho[2]) * (alpha[1] / omega[1]);
      b1 = beta[1];
      bo = -beta[1] * omega[1];
    }
    bDirection(c, A, init, b1, bo);
    init = false;
    bOp(c, A, A.v, A.pt, nullptr, 1);
    double m = bDot(c, A, A.rt, A.v, false);
    alpha[0] = rho[1] / m;
    if (fabs(m) > A.small * fabs(rho[1])) {
      const double a0 = alpha[0];
      norm[0] = bUpdateNorm(c, A, A.v, -a0, A.pt, a0, nullptr);
    } else {
      zeroV(A.r);
      norm[0] = 0.0;
    }
    if (norm[0] > A.eps * initial_norm && norm[0] > A.reps * initial_residual) {
      bPrecond(c, A, A.st, A.r);
      bOp(c, A, A.t, A.st, nullptr, 1);
      double tr, tt;
      bDot2(c, A, A.t, A.r, A.t, A.t, tr, tt);
      omega[0] = tr / tt;
      const double w0 = omega[0];
      norm[0] = bUpdateNorm(c, A, A.t, -w0, A.st, w0, &rhoNext);
      haveRho = true;
    }
    if (norm[0] <= A.eps * initial_norm || norm[0] <= A.reps * initial_residual) {
      status = 1;
      break;
    }
    if (omega[0] == 0.0 || norm[0] > (1 - A.hang) * norm[1]) {
      if (recount == 0) {
        recount = 1;
      } else {
        recount = 0;
        incrV(A.phi, A.e, 1.0);
        if (restarts == A.numRestarts) {
          if (c.tid() == 0) W.status[0] = 3, W.status[1] = iter;
          return;
        }
        bOp(c, A, A.r, A.phi, A.rhs, 0);
        norm[0] = bNormType(c, A, A.r);
        rho[1] = 0.0;
        rho[2] = 0.0;
        rho[3] = 0.0;
        alpha[0] = 0;
        beta[0] = 0;
        omega[0] = 0;
        restartVectors();
        haveRho = false;
        restarts++;
        init = true;
      }
    }
  }
  incrV(A.phi, A.e, 1.0);
  if (c.tid() == 0) W.status[0] = status, W.status[1] = iter;
}

template <class C>
__device__ void bottomRun(C& c, BottomArgs& A) {
  const BottomWork& W = A.W;
  A.r = W.v[0];
  A.rt = W.v[1];
  A.e = W.v[2];
  A.p = W.v[3];
  A.pt = W.v[4];
  A.st = W.v[5];
  A.t = W.v[6];
  A.v = W.v[7];
  A.phi = W.v[8];
  A.rhs = W.v[9];
  bCells(c, W.nv, [&](int q) {
    A.phi[q] = A.phiFab[W.fab[q]];
    A.rhs[q] = A.rhsFab[W.fab[q]];
  });
  if (A.cfg.kind == 1)
    bRelaxSolve(c, A);
  else
    bBicgstab(c, A);
  c.sync();
  for (int q = c.tid(); q < W.nv; q += c.nthr()) A.phiFab[W.fab[q]] = A.phi[q];
}

// One block per hierarchy of the level: block k solves with works[k] and
// metrics[k], the rest of the arguments shared.
__global__ void __launch_bounds__(1024) k_bottom(BottomArgs A0, const BottomWork* works, const double* metrics) {
  extern __shared__ double spart[];
  __shared__ double scal[8];
  BottomArgs A = A0;
  A.W = works[blockIdx.x];
  A.metric = metrics + blockIdx.x;
  if (A0.epsPer && A0.cfg.kind == 0) A.eps = A0.epsPer[blockIdx.x];
  BlkCtx c;
  c.part = spart;
  c.part2 = spart + max(A.W.nbox, 32);
  c.scal = scal;
  c.k = 0;
  bottomRun(c, A);
}

// One hierarchy, the whole grid (cooperative launch).
__global__ void __launch_bounds__(kBottomGridThreads) k_bottom_grid(BottomArgs A, const BottomWork* works,
                                                                    const double* metrics) {
  __shared__ double stage[2 * kBottomStage];
  A.W = works[0];
  A.metric = metrics;
  if (A.epsPer && A.cfg.kind == 0) A.eps = A.epsPer[0];
  GridCtx c;
  c.part = A.W.gpart;
  c.part2 = A.W.gpart2;
  c.scal = A.W.gscal;
  c.stage = stage;
  c.k = 0;
  bottomRun(c, A);
}

__global__ void k_gather_slots(const int* fab, int n, const double* src, double* dst) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) dst[q] = src[fab[q]];
}

}  // namespace

}  // namespace cmg

namespace cmg {

namespace {

Scal scalars(double dx, double alpha, double beta, int vc) {
  Scal s;
  s.dxinv = 1.0 / (dx * dx);
  double sum_b = 0.0;
  for (int d = 0; d < 3; ++d) sum_b = sum_b + 2.0 * s.dxinv;
  s.alpha = alpha;
  s.beta = beta;
  s.laplacian = (!vc && alpha == 0.0 && beta == 1.0) ? 1 : 0;
  s.lambda = s.laplacian ? -1.0 / sum_b : -1.0 / (alpha - beta * sum_b);
  return s;
}

}  // namespace

template <class T>
void ghostFill(const LevelDev& L, T* f, bool withCF, cudaStream_t s, int par) {
  auto range = [&](int p, int& r0, int& r1) {
    r0 = L.gcStart[p];
    r1 = r0 + L.gcExch[p] + (withCF ? L.gcCF[p] : 0);
  };
  int a0, a1, b0 = 0, b1 = 0;
  range(par >= 0 ? par : 0, a0, a1);
  if (par < 0) range(1, b0, b1);
  const int n = (a1 - a0) + (b1 - b0);
  if (n == 0) return;
  const double dx = L.dx, dxc = L.dxCrse;
  T c1 = T(2 * (dxc - dx) / (dxc + dx));
  T c2 = T(-(dxc - dx) / (dxc + 3 * dx));
  T flin = T(1 - 2 * dx / (dx + dxc));
  // Four entries per thread once the fill exceeds one wave of resident
  // threads (148 SMs x 2048), one per thread below that.
  if (n > 148 * 2048) {
    constexpr int U = 4;
    k_ghostcells<T, U><<<(n + GHOST_THREADS * U - 1) / (GHOST_THREADS * U), GHOST_THREADS, 0, s>>>(
        L.gcells, a0, a1, b0, b1, f, c1, c2, flin);
  } else {
    k_ghostcells<T, 1><<<(n + GHOST_THREADS - 1) / GHOST_THREADS, GHOST_THREADS, 0, s>>>(L.gcells, a0, a1, b0, b1, f,
                                                                                       c1, c2, flin);
  }
  CMG_LAUNCHED("ghostFill");
}

// BackwardEuler::createEulerRHS (BackwardEuler.cpp:190-226) over whole
// arrays: rhs = ((0 + phi) * a) + ((0 + src) * dt), a omitted for the
// constant-coefficient operator (its diagonalScale is a no-op).
__global__ void k_euler_rhs(double* rhs, const double* phi, const double* a, const double* src, double dt,
                            int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0 + phi[q];
    if (a) v = v * a[q];
    double w = 0.0 + src[q];
    w = w * dt;
    rhs[q] = v + w;
  }
}

// AMRTGA::oneStep's source term: (0 + src * 1) / a (setToZero, incr,
// divideByIdentityCoef; no division for the constant-coefficient operator).
__global__ void k_tga_source(double* out, const double* src, const double* a, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0 + src[q] * 1.0;
    if (a) v = v / a[q];
    out[q] = v;
  }
}

// x *= a (FArrayBox::mult by a FAB: the VC operator's diagonalScale).
__global__ void k_mult_field(double* x, const double* a, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    x[q] = x[q] * a[q];
}

void tgaSource(double* out, const double* src, const double* a, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  k_tga_source<<<flatBlocks(n), 256, 0, s>>>(out, src, a, n);
  CMG_LAUNCHED("tgaSource");
}

void multField(double* x, const double* a, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  k_mult_field<<<flatBlocks(n), 256, 0, s>>>(x, a, n);
  CMG_LAUNCHED("multField");
}

void eulerRHS(double* rhs, const double* phi, const double* a, const double* src, double dt, int64_t n,
              cudaStream_t s) {
  if (n == 0) return;
  k_euler_rhs<<<flatBlocks(n), 256, 0, s>>>(rhs, phi, a, src, dt, n);
  CMG_LAUNCHED("eulerRHS");
}

void scaleField(double* x, double scale, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  k_scale_flat<<<flatBlocks(n), 256, 0, s>>>(x, scale, n);
  CMG_LAUNCHED("scale");
}

void boxDots(const LevelDev& L, const double* x, const double* y, double* out, cudaStream_t s) {
  if (L.nbox == 0) return;
  k_box_dot<<<L.nbox, 32, 0, s>>>(L.boxes, x, y, out);
  CMG_LAUNCHED("boxDots");
}

template <class T>
void zeroCovered(const LevelDev& L, T* f, cudaStream_t s) {
  if (L.nZero == 0) return;
  k_ghost<T><<<(L.nCellsZero + GHOST_PER_BLOCK - 1) / GHOST_PER_BLOCK, GHOST_THREADS, 0, s>>>(
      L.zero, L.zeroStart, L.zeroBlock, L.nZero, L.nCellsZero, -1, f, T(0), T(0), T(0));
  CMG_LAUNCHED("zeroCovered");
}

template <class T>
void relaxBlock(const LevelDev& L, T* phi, const T* rhs, const Coef<T>& c, int nsweeps, cudaStream_t s) {
  if (L.nColor[0] + L.nColor[1] == 0 || nsweeps <= 0) return;
  Scal sc = scalars(L.dx, c.alpha, c.beta, c.vc);
  const double dx = L.dx, dxc = L.dxCrse;
  GhostCoef gc{2 * (dxc - dx) / (dxc + dx), -(dxc - dx) / (dxc + 3 * dx), 1 - 2 * dx / (dx + dxc)};
  if (c.vc)
    k_relax_block<T, 1><<<1, 1024, 0, s>>>(L.boxes, L.chColor[0], L.nColor[0], L.chColor[1], L.nColor[1], phi, rhs,
                                           sc, c.a, c.b[0], c.b[1], c.b[2], c.lambda, L.faceRules, L.faceOff, gc,
                                           nsweeps);
  else
    k_relax_block<T, 0><<<1, 1024, 0, s>>>(L.boxes, L.chColor[0], L.nColor[0], L.chColor[1], L.nColor[1], phi, rhs,
                                           sc, nullptr, nullptr, nullptr, nullptr, nullptr, L.faceRules, L.faceOff,
                                           gc, nsweeps);
  CMG_LAUNCHED("relaxBlock");
}

template <class T>
void gsrb(const LevelDev& L, T* phi, const T* rhs, const Coef<T>& c, int color, cudaStream_t s, bool inlineGhosts) {
  int n = L.nColor[color];
  if (n == 0) return;
  Scal sc = scalars(L.dx, c.alpha, c.beta, c.vc);
  const double dx = L.dx, dxc = L.dxCrse;
  GhostCoef gc{2 * (dxc - dx) / (dxc + dx), -(dxc - dx) / (dxc + 3 * dx), 1 - 2 * dx / (dx + dxc)};
  auto launch = [&](auto kern, const T* a, const T* b0, const T* b1, const T* b2, const T* lam) {
    kern<<<n, CHUNK, 0, s>>>(L.boxes, L.chColor[color], phi, rhs, color, sc, a, b0, b1, b2, lam,
                             L.chGhost[color], L.chGhostStart[color], gc);
  };
  auto launchPair = [&](auto kern, const T* a, const T* b0, const T* b1, const T* b2, const T* lam) {
    kern<<<n, CHUNK / 2, 0, s>>>(L.boxes, L.chColor[color], phi, rhs, color, sc, a, b0, b1, b2, lam);
  };
  if (c.vc) {
    if (inlineGhosts)
      launch(k_gsrb<T, 1, true>, c.a, c.b[0], c.b[1], c.b[2], c.lambda);
    else
      launchPair(k_gsrb_pair<T, 1>, c.a, c.b[0], c.b[1], c.b[2], c.lambda);
  } else {
    if (inlineGhosts)
      launch(k_gsrb<T, 0, true>, nullptr, nullptr, nullptr, nullptr, nullptr);
    else
      launchPair(k_gsrb_pair<T, 0>, nullptr, nullptr, nullptr, nullptr, nullptr);
  }
  CMG_LAUNCHED("gsrb");
}

template <class T>
void gsrbSweepFused(const LevelDev& L, T* phi, const T* rhs, const Coef<T>& c, cudaStream_t s) {
  if (L.nbox == 0) return;
  Scal sc = scalars(L.dx, c.alpha, c.beta, c.vc);
  const double dx = L.dx, dxc = L.dxCrse;
  GhostCoef gc{2 * (dxc - dx) / (dxc + dx), -(dxc - dx) / (dxc + 3 * dx), 1 - 2 * dx / (dx + dxc)};
  const int nd = L.nDeferred, db = (nd + 255) / 256;
  if (c.vc) {
    k_gsrb_march<T, 1><<<L.nbox, 256, 0, s>>>(L.boxes, phi, rhs, sc, c.a, c.b[0], c.b[1], c.b[2], c.lambda,
                                              L.faceRules, L.faceOff, gc);
    CMG_LAUNCHED("gsrbMarch");
    if (nd > 0) {
      k_gsrb_deferred<T, 1><<<db, 256, 0, s>>>(L.boxes, L.deferred, nd, phi, rhs, sc, c.a, c.b[0], c.b[1], c.b[2],
                                               c.lambda, L.faceRules, L.faceOff, gc);
      CMG_LAUNCHED("gsrbDeferred");
    }
  } else {
    k_gsrb_march<T, 0><<<L.nbox, 256, 0, s>>>(L.boxes, phi, rhs, sc, nullptr, nullptr, nullptr, nullptr, nullptr,
                                              L.faceRules, L.faceOff, gc);
    CMG_LAUNCHED("gsrbMarch");
    if (nd > 0) {
      k_gsrb_deferred<T, 0><<<db, 256, 0, s>>>(L.boxes, L.deferred, nd, phi, rhs, sc, nullptr, nullptr, nullptr,
                                               nullptr, nullptr, L.faceRules, L.faceOff, gc);
      CMG_LAUNCHED("gsrbDeferred");
    }
  }
}

template <class T>
void residual(const LevelDev& L, T* r, const T* phi, const T* rhs, const Coef<T>& c, cudaStream_t s) {
  if (L.nAll == 0) return;
  Scal sc = scalars(L.dx, c.alpha, c.beta, c.vc);
  const int n = L.nColor[0];
  if (c.vc)
    k_op_pair<T, 1, 0><<<n, CHUNK, 0, s>>>(L.boxes, L.chColor[0], L.chColor[1], r, phi, rhs, sc, c.a, c.b[0],
                                           c.b[1], c.b[2]);
  else
    k_op_pair<T, 0, 0><<<n, CHUNK, 0, s>>>(L.boxes, L.chColor[0], L.chColor[1], r, phi, rhs, sc, nullptr, nullptr,
                                           nullptr, nullptr);
  CMG_LAUNCHED("residual");
}

template <class T>
void applyOp(const LevelDev& L, T* lofphi, const T* phi, const Coef<T>& c, cudaStream_t s) {
  if (L.nAll == 0) return;
  Scal sc = scalars(L.dx, c.alpha, c.beta, c.vc);
  const int n = L.nColor[0];
  if (c.vc)
    k_op_pair<T, 1, 1><<<n, CHUNK, 0, s>>>(L.boxes, L.chColor[0], L.chColor[1], lofphi, phi, nullptr, sc, c.a,
                                           c.b[0], c.b[1], c.b[2]);
  else
    k_op_pair<T, 0, 1><<<n, CHUNK, 0, s>>>(L.boxes, L.chColor[0], L.chColor[1], lofphi, phi, nullptr, sc, nullptr,
                                           nullptr, nullptr, nullptr);
  CMG_LAUNCHED("applyOp");
}

template <class T>
void negAdd(const LevelDev& L, T* r, const T* lofphi, const T* rhs, cudaStream_t s) {
  if (L.nelem == 0) return;
  k_negadd_flat<T><<<flatBlocks(L.nelem), 256, 0, s>>>(r, lofphi, rhs, L.nelem);
  CMG_LAUNCHED("negAdd");
}

template <class T>
void restrictMG(const LevelDev& F, const LevelDev& C, T* resC, const T* phi, const T* rhs, const Coef<T>& c,
                cudaStream_t s) {
  if (C.nAll == 0) return;
  Scal sc = scalars(F.dx, c.alpha, c.beta, c.vc);
  if (c.vc)
    k_restrictmg<T, 1><<<C.nAll, CHUNK, 0, s>>>(F.boxes, C.boxes, C.chAll, resC, phi, rhs, sc, c.a, c.b[0], c.b[1],
                                                c.b[2]);
  else
    k_restrictmg<T, 0><<<C.nAll, CHUNK, 0, s>>>(F.boxes, C.boxes, C.chAll, resC, phi, rhs, sc, nullptr, nullptr,
                                                nullptr, nullptr);
  CMG_LAUNCHED("restrictMG");
}

template <class T>
void prolongMG(const LevelDev& F, const LevelDev& C, T* phi, const T* corrC, cudaStream_t s) {
  if (F.nAll == 0) return;
  k_prolongmg<T><<<F.nAll, CHUNK, 0, s>>>(F.boxes, C.boxes, F.chAll, phi, corrC);
  CMG_LAUNCHED("prolongMG");
}

template <class T>
void averageAMR(const LevelDev& F, const LevelDev& C, T* coarse, const T* fine, cudaStream_t s) {
  if (F.nItemChC == 0) return;
  k_average<T><<<F.nItemChC, CHUNK, 0, s>>>(F.boxes, C.boxes, F.items, F.itemChC, coarse, fine);
  CMG_LAUNCHED("averageAMR");
}

template <class T>
void prolongAMR(const LevelDev& F, const LevelDev& C, T* fine, const T* coarse, cudaStream_t s) {
  if (F.nItemChF == 0) return;
  k_prolongamr<T><<<F.nItemChC, CHUNK, 0, s>>>(F.boxes, C.boxes, F.items, F.itemChC, fine, coarse);
  CMG_LAUNCHED("prolongAMR");
}

template <class T>
void quadCF(const LevelDev& F, T* phiF, const T* phiC, cudaStream_t s) {
  if (F.nCfF == 0) return;
  T* tmp = reinterpret_cast<T*>(F.cfTmp);
  k_cf_coarse<T><<<(F.nCfC + 127) / 128, 128, 0, s>>>(F.cfC, F.nCfC, F.cfW, F.cfOff, phiC, T(F.dx), tmp);
  CMG_LAUNCHED("quadCFCoarse");
  k_quadcf<T><<<(F.nCfF + 127) / 128, 128, 0, s>>>(F.cfF, F.nCfF, tmp, phiF, T(F.dx));
  CMG_LAUNCHED("quadCF");
}

template <class T>
void reflux(const LevelDev& C, T* lofphiC, const T* phiC, const T* phiF, const Coef<T>& cc, const Coef<T>& cf,
            cudaStream_t s) {
  if (C.nRf == 0) return;
  int nb = (C.nRf + 127) / 128;
  // getFlux scale beta * ref / dx with the coarse dx (AMRPoissonOp.cpp:1797-1851).
  T sc = T(cc.beta * 1 / C.dx);
  T sf = T(cc.beta * 2 / C.dx);
  T negs = T(-(1.0 / C.dx));
  if (cc.vc)
    k_reflux<T, 1><<<nb, 128, 0, s>>>(C.rfCells, C.nRf, C.rfC, C.rfF, lofphiC, phiC, phiF, cc.b[0], cc.b[1],
                                      cc.b[2], cf.b[0], cf.b[1], cf.b[2], sc, sf, negs);
  else
    k_reflux<T, 0><<<nb, 128, 0, s>>>(C.rfCells, C.nRf, C.rfC, C.rfF, lofphiC, phiC, phiF, nullptr, nullptr,
                                      nullptr, nullptr, nullptr, nullptr, sc, sf, negs);
  CMG_LAUNCHED("reflux");
}

template <class T>
void incr(const LevelDev& L, T* lhs, const T* x, double scale, cudaStream_t s) {
  if (L.nelem == 0) return;
  k_incr_flat<T, T><<<flatBlocks(L.nelem), 256, 0, s>>>(lhs, x, T(scale), L.nelem);
  CMG_LAUNCHED("incr");
}

template <class T>
void incrCopy(const LevelDev& L, T* lhs, T* x, cudaStream_t s) {
  if (L.nelem == 0) return;
  k_incr_copy_flat<T><<<flatBlocks(L.nelem), 256, 0, s>>>(lhs, x, L.nelem);
  CMG_LAUNCHED("incrCopy");
}

template <class T>
void incrZero(const LevelDev& L, T* lhs, T* x, cudaStream_t s) {
  if (L.nelem == 0) return;
  k_incr_zero_flat<T><<<flatBlocks(L.nelem), 256, 0, s>>>(lhs, x, L.nelem);
  CMG_LAUNCHED("incrZero");
}

template <class T>
void maxNorm(const LevelDev& L, const T* f, double* out, cudaStream_t s) {
  if (L.nAll == 0) return;
  if (L.boxHier) {
    k_maxnorm_hier<T><<<L.nAll, CHUNK, 0, s>>>(L.boxes, L.chAll, L.boxHier, f, out);
    CMG_LAUNCHED("maxNorm");
    return;
  }
  // One chunk per block (lowest latency) up to 4096 chunks; beyond, a
  // grid of 4096 blocks striding over them.
  const int blocks = std::min(L.nAll, 4096);
  k_maxnorm<T><<<blocks, CHUNK, 0, s>>>(L.boxes, L.chAll, L.nAll, f, out);
  CMG_LAUNCHED("maxNorm");
}


long long launchCount() { return g_launches.load(std::memory_order_relaxed); }
void addLaunches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void bottomSolve(const LevelDev& L, double* phi, const double* rhs, const Coef<double>& c, const BottomWork* works,
                 int nworks, int maxBoxes, const BottomConfig& cfg, double eps, const double* metrics,
                 cudaStream_t s, const double* epsPer, int gridBlocks) {
  if (nworks == 0) return;
  BottomArgs A;
  A.boxes = L.boxes;
  A.sc = scalars(L.dx, c.alpha, c.beta, c.vc);
  A.vc = c.vc;
  A.phiFab = phi;
  A.rhsFab = rhs;
  A.cfg = cfg;
  A.eps = cfg.kind == 1 ? cfg.eps : eps;  // RelaxSolver keeps its own tolerance
  A.epsPer = epsPer;
  A.reps = cfg.reps;
  A.hang = cfg.hang;
  A.small = cfg.small;
  A.imax = cfg.imax;
  A.numRestarts = cfg.numRestarts;
  // AMRPoissonOp::preCond multiplier (AMRPoissonOp.cpp:304-329).
  A.mult = 1.0 / (c.alpha - 2.0 * 3 * c.beta / (L.dx * L.dx));
  if (gridBlocks > 0) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(gridBlocks);
    lc.blockDim = dim3(kBottomGridThreads);
    lc.dynamicSmemBytes = 0;
    lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    check(cudaLaunchKernelEx(&lc, k_bottom_grid, A, works, metrics), "bottomSolve (grid)");
    CMG_LAUNCHED("bottomSolve");
    return;
  }
  const size_t smem = 2 * (size_t)std::max(maxBoxes, 32) * sizeof(double);
  if (smem > 48 * 1024) {
    if (smem > 200 * 1024) throw std::runtime_error("cmg: bottom level with too many boxes for one block");
    check(cudaFuncSetAttribute(k_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "bottom smem");
  }
  k_bottom<<<nworks, 1024, smem, s>>>(A, works, metrics);
  CMG_LAUNCHED("bottomSolve");
}

int bottomGridBlocks(int nv) {
  int dev = 0, sms = 0, occ = 0;
  check(cudaGetDevice(&dev), "device");
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bottom_grid, kBottomGridThreads, 0), "occupancy");
  const int want = (nv + kBottomGridThreads - 1) / kBottomGridThreads;
  return std::max(1, std::min(want, sms * std::max(occ, 1)));
}

int bottomGridThreads() { return kBottomGridThreads; }

void gatherSlots(const BottomWork& w, const double* fab, double* dst, cudaStream_t s) {
  const int n = w.nv + w.ng;
  if (n == 0) return;
  k_gather_slots<<<(n + 255) / 256, 256, 0, s>>>(w.fab, n, fab, dst);
  CMG_LAUNCHED("gatherSlots");
}

void incrMixed(const LevelDev& L, double* lhs, const float* x, cudaStream_t s) {
  if (L.nelem == 0) return;
  k_incr_flat<double, float><<<flatBlocks(L.nelem), 256, 0, s>>>(lhs, x, 1.0, L.nelem);
  CMG_LAUNCHED("incrMixed");
}

template <class T, class X>
void incrActive(const LevelDev& L, T* lhs, const X* x, const int* active, cudaStream_t s) {
  if (L.nelem == 0) return;
  const int64_t per = (L.nelem + L.nh - 1) / L.nh;
  const int bx = (int)std::max<int64_t>(1, std::min<int64_t>((per + 255) / 256, 64));
  k_incr_active<T, X><<<dim3(bx, L.nh), 256, 0, s>>>(lhs, x, L.hierStart, active);
  CMG_LAUNCHED("incrActive");
}
template void incrActive<double, double>(const LevelDev&, double*, const double*, const int*, cudaStream_t);
template void incrActive<double, float>(const LevelDev&, double*, const float*, const int*, cudaStream_t);

template <class D, class S>
void convert(D* dst, const S* src, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_convert<D, S><<<blocks, 256, 0, s>>>(dst, src, n);
  CMG_LAUNCHED("convert");
}
template void convert<float, double>(float*, const double*, int64_t, cudaStream_t);
template void convert<double, float>(double*, const float*, int64_t, cudaStream_t);

// ------------------------------------------------ synthetic inputs, device
// The seeded fields of synthetic.H evaluated on the device (same formulas and
// operation order; exp and cos of the CUDA math library, so values agree with
// the host generator to within their last bits), and the coefficient set-up
// of finalizeCoefficients (resetLambda with SUMFACES, MG coefficient
// averages) with the host code's operation order.
namespace {

__global__ void k_fill_cells(const BoxDesc* boxes, const Chunk* chunks, double dx, cmg_synth::Bumps bumps,
                             cmg_synth::Modes am, double* rhs, double* a) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  int i, j, k;
  if (!allCell(bd, ch.start + threadIdx.x, i, j, k)) return;
  const double x = (i + 0.5) * dx, y = (j + 0.5) * dx, z = (k + 0.5) * dx;
  const int64_t c = cellIndex(bd, i, j, k);
  rhs[c] = devBumps(bumps, x, y, z);
  if (a) a[c] = devModes(am, x, y, z);
}

// One block per box: faces lo..hi+1 in direction d.
__global__ void k_fill_faces(const BoxDesc* boxes, double dx, int d, cmg_synth::Modes bm, double* b) {
  const BoxDesc bd = boxes[blockIdx.x];
  int n[3];
  for (int e = 0; e < 3; ++e) n[e] = bd.hi[e] - bd.lo[e] + 1 + (e == d);
  const int total = n[0] * n[1] * n[2];
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    int iv[3] = {bd.lo[0] + q % n[0], bd.lo[1] + (q / n[0]) % n[1], bd.lo[2] + q / (n[0] * n[1])};
    double x[3];
    for (int e = 0; e < 3; ++e) x[e] = (e == d) ? iv[e] * dx : (iv[e] + 0.5) * dx;
    b[cellIndex(bd, iv[0], iv[1], iv[2])] = devModes(bm, x[0], x[1], x[2]);
  }
}

// lambda = 1 / (alpha a + sum_d scale beta (b_hi + b_lo)) (computeLambda).
__global__ void k_lambda(const BoxDesc* boxes, const Chunk* chunks, const double* a, const double* b0,
                         const double* b1, const double* b2, double alpha, double beta, double dx, double* lam) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc bd = boxes[ch.box];
  int i, j, k;
  if (!allCell(bd, ch.start + threadIdx.x, i, j, k)) return;
  const Stencil st = stencil(bd, i, j, k);
  const double scale = 1.0 / (dx * dx);
  double l = a[st.c] * alpha;
  l = l + scale * beta * (b0[st.xp] + b0[st.c]);
  l = l + scale * beta * (b1[st.yp] + b1[st.c]);
  l = l + scale * beta * (b2[st.zp] + b2[st.c]);
  lam[st.c] = 1.0 / l;
}

// averageCells: coarse(i) = refScale * sum of its r^3 fine values in k-j-i order.
__global__ void k_avg_cells(const BoxDesc* fboxes, const BoxDesc* cboxes, const Chunk* chunks, int r,
                            const double* f, double* out) {
  Chunk ch = chunks[blockIdx.x];
  const BoxDesc cb = cboxes[ch.box];
  int i, j, k;
  if (!allCell(cb, ch.start + threadIdx.x, i, j, k)) return;
  const BoxDesc fb = fboxes[ch.box];
  const double refScale = 1.0 / (double)(r * r * r);
  double s = 0.0;
  bool first = true;
  for (int c = 0; c < r; ++c)
    for (int bb = 0; bb < r; ++bb)
      for (int aa = 0; aa < r; ++aa) {
        double v = f[cellIndex(fb, i * r + aa, j * r + bb, k * r + c)];
        s = first ? v : s + v;
        first = false;
      }
  out[cellIndex(cb, i, j, k)] = refScale * s;
}

// averageFaces: coarse face = refScale * sum over the r^2 fine faces.
__global__ void k_avg_faces(const BoxDesc* fboxes, const BoxDesc* cboxes, int r, int d, const double* f,
                            double* out) {
  const BoxDesc cb = cboxes[blockIdx.x];
  const BoxDesc fb = fboxes[blockIdx.x];
  int n[3], ext[3] = {r, r, r};
  ext[d] = 1;
  for (int e = 0; e < 3; ++e) n[e] = cb.hi[e] - cb.lo[e] + 1 + (e == d);
  const double base = 1.0 / (double)r;
  const double refScale = base * base;
  const int total = n[0] * n[1] * n[2];
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    int i = cb.lo[0] + q % n[0], j = cb.lo[1] + (q / n[0]) % n[1], k = cb.lo[2] + q / (n[0] * n[1]);
    double s = 0;
    for (int c = 0; c < ext[2]; ++c)
      for (int bb = 0; bb < ext[1]; ++bb)
        for (int aa = 0; aa < ext[0]; ++aa) s = s + f[cellIndex(fb, i * r + aa, j * r + bb, k * r + c)];
    out[cellIndex(cb, i, j, k)] = refScale * s;
  }
}

}  // namespace

void fillSyntheticLevel(const LevelDev& L, uint64_t seed, double* rhs, double* a, double* const b[3],
                        cudaStream_t s) {
  fillSyntheticBoxes(L, seed, rhs, a, b, 0, L.nbox, 0, L.nAll, s);
}

void fillSyntheticBoxes(const LevelDev& L, uint64_t seed, double* rhs, double* a, double* const b[3], int box0,
                        int box1, int ch0, int ch1, cudaStream_t s) {
  cmg_synth::Problem prob(seed);
  if (ch1 <= ch0) return;
  k_fill_cells<<<ch1 - ch0, CHUNK, 0, s>>>(L.boxes, L.chAll + ch0, L.dx, prob.bumps, prob.acoef, rhs, a);
  CMG_LAUNCHED("fillCells");
  if (!b || box1 <= box0) return;
  for (int d = 0; d < 3; ++d) {
    k_fill_faces<<<box1 - box0, 256, 0, s>>>(L.boxes + box0, L.dx, d, prob.bcoef, b[d]);
    CMG_LAUNCHED("fillFaces");
  }
}

void lambdaLevel(const LevelDev& L, const double* a, const double* const b[3], double alpha, double beta,
                 double* lam, cudaStream_t s) {
  if (L.nAll == 0) return;
  k_lambda<<<L.nAll, CHUNK, 0, s>>>(L.boxes, L.chAll, a, b[0], b[1], b[2], alpha, beta, L.dx, lam);
  CMG_LAUNCHED("lambda");
}

void averageCoefficients(const LevelDev& F, const LevelDev& C, int r, const double* fa, const double* const fb[3],
                         double* ca, double* const cbf[3], cudaStream_t s) {
  if (C.nAll == 0) return;
  k_avg_cells<<<C.nAll, CHUNK, 0, s>>>(F.boxes, C.boxes, C.chAll, r, fa, ca);
  CMG_LAUNCHED("averageCells");
  for (int d = 0; d < 3; ++d) {
    k_avg_faces<<<C.nbox, 256, 0, s>>>(F.boxes, C.boxes, r, d, fb[d], cbf[d]);
    CMG_LAUNCHED("averageFaces");
  }
}

#define CMG_INST(T)                                                                                       \
  template void ghostFill<T>(const LevelDev&, T*, bool, cudaStream_t, int);                                \
  template void zeroCovered<T>(const LevelDev&, T*, cudaStream_t);                                         \
  template void gsrb<T>(const LevelDev&, T*, const T*, const Coef<T>&, int, cudaStream_t, bool);           \
  template void relaxBlock<T>(const LevelDev&, T*, const T*, const Coef<T>&, int, cudaStream_t);              \
  template void gsrbSweepFused<T>(const LevelDev&, T*, const T*, const Coef<T>&, cudaStream_t);            \
  template void residual<T>(const LevelDev&, T*, const T*, const T*, const Coef<T>&, cudaStream_t);        \
  template void applyOp<T>(const LevelDev&, T*, const T*, const Coef<T>&, cudaStream_t);                   \
  template void negAdd<T>(const LevelDev&, T*, const T*, const T*, cudaStream_t);                          \
  template void restrictMG<T>(const LevelDev&, const LevelDev&, T*, const T*, const T*, const Coef<T>&,    \
                              cudaStream_t);                                                               \
  template void prolongMG<T>(const LevelDev&, const LevelDev&, T*, const T*, cudaStream_t);                \
  template void averageAMR<T>(const LevelDev&, const LevelDev&, T*, const T*, cudaStream_t);               \
  template void prolongAMR<T>(const LevelDev&, const LevelDev&, T*, const T*, cudaStream_t);               \
  template void quadCF<T>(const LevelDev&, T*, const T*, cudaStream_t);                                    \
  template void reflux<T>(const LevelDev&, T*, const T*, const T*, const Coef<T>&, const Coef<T>&,         \
                          cudaStream_t);                                                                   \
  template void incrCopy<T>(const LevelDev&, T*, T*, cudaStream_t);                                         \
  template void incrZero<T>(const LevelDev&, T*, T*, cudaStream_t);                                         \
  template void incr<T>(const LevelDev&, T*, const T*, double, cudaStream_t);                              \
  template void maxNorm<T>(const LevelDev&, const T*, double*, cudaStream_t);

CMG_INST(double)
CMG_INST(float)

}  // namespace cmg
