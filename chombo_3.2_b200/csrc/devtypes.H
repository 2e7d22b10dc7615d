// Plain-old-data tables that the host plan builder writes and the CUDA
// kernels read.  One level's fields all share one ghosted layout:
//   every box owns a FAB of px x (ny+2) x (nz+2) cells (one ghost layer;
//   px = nx+2 rounded up to even), stored red-black ordered: the cells of
//   colour 0 ((i+j+k) even) first, then those of colour 1, each half in
//   x-fastest order of the FAB with two x-neighbours sharing one slot.  A
//   red-black pass therefore touches only its own colour's half of every
//   cell-centred array (plus the other colour's phi), with contiguous,
//   coalesced rows, and never moves bytes of the colour it does not update.
// Face-centred data (the b coefficient in direction d) uses the same layout:
// the face on the low side of cell i in direction d is stored at cell i, so
// faces lo..hi+1 fit in the valid region plus the high ghost layer.
#ifndef CMG_DEVTYPES_H
#define CMG_DEVTYPES_H

#include <stdint.h>

namespace cmg {

struct BoxDesc {
  int lo[3], hi[3];
  int px, py;       // x pitch (even) and y extent (ny + 2) of the ghosted FAB
  int64_t off;      // element offset of the box's FAB
  int64_t half;     // elements per colour (px * py * (nz + 2) / 2)
  // Division multipliers (divMagic) for the cell enumerations: by nx, by
  // (nx + 1) / 2 and by ny; 0 where a box is too large for them (a plain
  // division is used there).
  uint64_t mNx, mHalf, mNy;
};

#if defined(__CUDACC__)
#define CMG_HD __host__ __device__ __forceinline__
#else
#define CMG_HD inline
#endif

// ceil(2^32 / d): for 0 <= q < 2^32 / d, q / d == (q * divMagic(d)) >> 32
// (the rounding error of the multiplier, below d, cannot carry into the
// integer part for such q), which replaces the divide sequence of a runtime
// divisor by one wide multiply.  qmax: the largest dividend; 0 (plain
// division) when it is outside that range.
CMG_HD uint64_t divMagic(int d, int64_t qmax) {
  if (d < 1 || qmax < 0 || (uint64_t)qmax >= (uint64_t(1) << 32) / (uint64_t)d) return 0;
  return ((uint64_t(1) << 32) + (uint64_t)d - 1) / (uint64_t)d;
}
CMG_HD int fastDiv(int q, int d, uint64_t m) {
  return m ? (int)(((uint64_t)(unsigned)q * m) >> 32) : q / d;
}

// Slot of cell (i,j,k) within its colour half (x-neighbour pairs share it).
CMG_HD int64_t colourSlot(const BoxDesc& b, int i, int j, int k) {
  return ((int64_t)(i - b.lo[0] + 1) + (int64_t)b.px * ((int64_t)(j - b.lo[1] + 1) + (int64_t)b.py * (k - b.lo[2] + 1))) >> 1;
}

CMG_HD int64_t cellIndex(const BoxDesc& b, int i, int j, int k) {
  return b.off + ((i + j + k) & 1) * b.half + colourSlot(b, i, j, k);
}

// Element indices of a cell and of its six face neighbours (a level holds
// fewer than 2^31 elements, which the plan builder checks).
struct Stencil {
  int c, xp, xm, yp, ym, zp, zm;
};

CMG_HD Stencil stencil(const BoxDesc& b, int i, int j, int k) {
  Stencil s;
  const int col = (i + j + k) & 1;
  const int m = ((i - b.lo[0] + 1) + b.px * ((j - b.lo[1] + 1) + b.py * (k - b.lo[2] + 1))) >> 1;
  const int off = (int)b.off, half = (int)b.half;
  const int own = off + col * half, oth = off + (1 - col) * half + m;
  const int xo = (i - b.lo[0] + 1) & 1;  // x parity inside the FAB
  const int sy = b.px >> 1, sz = (b.px >> 1) * b.py;
  s.c = own + m;
  s.xp = oth + xo;
  s.xm = oth + xo - 1;
  s.yp = oth + sy;
  s.ym = oth - sy;
  s.zp = oth + sz;
  s.zm = oth - sz;
  return s;
}

// Ghost-layer work items executed by one kernel per fill (exchange copies,
// physical boundary values, homogeneous coarse-fine values, zeroing).
enum GhostKind {
  G_COPY = 0,      // dst(cell) = src(cell), cells of region (Copier item)
  G_BC = 1,        // homogeneous first-order Dirichlet: g = 2*0 - interior
  G_CFQUAD = 2,    // homogeneous quadratic CF: g = c1*phi(1 in) + c2*phi(2 in)
  G_CFLIN = 3,     // one-cell-wide box: g = f*phi(1 in)
  G_ZERO = 4,      // dst(cell) = 0 (covered cells before a norm)
  G_NEU = 5        // homogeneous Neumann: g = interior (NeumBC, BCFunc.cpp:217-236)
};

// Ghost cells handled by one thread block of the ghost kernel (each thread
// takes GHOST_PER_THREAD of them, GHOST_THREADS apart).
enum { GHOST_THREADS = 256, GHOST_PER_THREAD = 1, GHOST_PER_BLOCK = GHOST_THREADS * GHOST_PER_THREAD };

struct GhostTask {
  int kind, dst, src, dir, side;  // side = -1 (low) or +1 (high)
  int lo[3], hi[3];
  int shift[3];  // exchange from a periodic image: the source cell is (i,j,k) - shift
};

// One ghost cell of a level's ghost fill, as element indices: dst = src1
// (s2 == -1, exchange copy or homogeneous Neumann face), dst = 2*0 - src1
// (s2 == -2, homogeneous
// Dirichlet face), dst = flin*src1 (s2 == -3, linear coarse-fine ghost of a
// one-cell-wide box), dst = c1*src1 + c2*s2 (s2 >= 0, quadratic coarse-fine).
struct GhostCell {
  int dst, s1, s2;
};

// How a relaxation pass obtains the value of one face-ghost cell of a box
// without a ghost fill: the rule the fill before the pass would apply,
// evaluated at the moment the adjacent valid cell (the only cell whose
// stencil reads this ghost) is updated.  Every value the rule reads belongs to
// the other colour or is the updated cell's own old value, so it is the value
// the fill would have written.
enum FaceRuleKind {
  FR_COPY = 0,    // exchange: src = element of the source box's valid cell
  FR_BC = 1,      // homogeneous Dirichlet: 2*0 - (the adjacent cell)
  FR_CFQUAD = 2,  // homogeneous quadratic CF: c1*(adjacent) + c2*f[src], src two cells inward
  FR_CFLIN = 3,   // linear CF of a one-cell-wide box: flin*(adjacent)
  FR_FAB = 4,     // no fill rule: the FAB ghost element src as it is
  FR_NEU = 5      // homogeneous Neumann: the adjacent cell itself
};
struct FaceRule {
  int src, kind;
};

// A colour-1 cell of a box that lies on a face whose ghost is an exchange
// copy from another box (FR_COPY rule): the fused red-black sweep (one launch
// per sweep, every box marching through its z slabs) cannot update it before
// every box has finished its colour-0 cells, so a second launch does, from
// this list.  q: the cell's index in its box, x fastest.
struct DeferredCell {
  int box, q;
};

// Device form of a ghost task: the task plus copies of its destination and
// source box descriptors, so that a thread reaches its data after a single
// table load.
struct GhostTaskDev {
  BoxDesc dst, src;
  int kind, dir, side;
  int lo[3], hi[3];
  int shift[3];  // GhostTask::shift
  int ax;  // one-colour enumeration steps by 2 along this axis (first with extent > 1)
};

// Slots of a task in a one-colour fill: ceil(n_ax / 2) per line along ax.
CMG_HD int64_t colourSlots(const int lo[3], const int hi[3], int ax) {
  int64_t n = 1;
  for (int d = 0; d < 3; ++d) n *= d == ax ? (hi[d] - lo[d] + 2) / 2 : (hi[d] - lo[d] + 1);
  return n;
}
CMG_HD int parityAxis(const int lo[3], const int hi[3]) {
  return hi[0] > lo[0] ? 0 : hi[1] > lo[1] ? 1 : hi[2] > lo[2] ? 2 : 0;
}

// Work decomposition of a box list into fixed-size chunks of cells (or of
// one colour's cells for red-black sweeps): chunk c covers cells
// [start, start + CHUNK) of box `box` in the enumeration used by the kernel.
struct Chunk {
  int box;
  int start;
};

// Inhomogeneous quadratic coarse-fine interpolation (QuadCFInterp): one entry
// per fine ghost cell.  Coarse data are read straight from the coarse level
// through precomputed element offsets.
struct CFDeriv {
  int kind;   // 0: zero, 1: centred standard form, 2: weighted stencil
  int n;      // number of (weight, offset) pairs for kind 2
  int start;  // first pair in the pool; kind 1 uses pool offsets only
};
struct CFCoarse {
  int64_t cc;      // offset of the coarse cell under the ghost
  CFDeriv d1[2];   // first derivatives along the two tangential directions
  CFDeriv d2[2];   // second derivatives
  CFDeriv mx;      // mixed derivative
};
struct CFFine {
  int64_t g;       // fine ghost cell
  int64_t pa, pb;  // fine cells 2 and 1 inward of the ghost
  double x1, x2;   // tangential offsets of the fine centre from the coarse centre
  int coarse;      // CFCoarse index
  int packed;      // 1: Fortran-form interpolation, 0: C++-form
};

// Flux-register correction of one uncovered coarse cell next to finer cells.
struct RefluxCell {
  int64_t c;       // coarse cell (coarse level layout)
  int nco;         // coarse face terms (<= 6)
  int nfi;         // fine face groups (<= 6), each of 4 fine faces
  int start;       // first coarse term in the term pool
  int fstart;      // first fine group in the group pool
};
struct RefluxCoarseTerm {
  int64_t hi, lo;  // cells on each side of the coarse face
  int64_t bface;   // face coefficient element (VC), -1 otherwise
  int dir;
  double sgn;      // +1 (low-side location) or -1 (high-side)
};
struct RefluxFineGroup {
  int64_t hi[4], lo[4];  // cells on each side of the 4 fine faces, k-j-i order
  int64_t bface[4];
  int dir;
  double scale;          // sign(side) * 1 / nRef^2
};

// Map between a fine level and its coarse parent: one item per (coarse box,
// fine box) pair whose coarsened fine box meets the coarse box; region is in
// coarse index space.
struct CoarseFineItem {
  int cbox, fbox;
  int lo[3], hi[3];
};

}  // namespace cmg

#endif
