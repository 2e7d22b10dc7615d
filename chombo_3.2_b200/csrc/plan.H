// Host-side plans for one hierarchy: per-level box tables, ghost work lists,
// red-black work chunks, coarse-fine interpolation stencils, flux-register
// correction lists and coarse-fine box maps.  Everything here is built once
// per hierarchy shape and uploaded; the V-cycle only reads it.
#ifndef CMG_PLAN_H
#define CMG_PLAN_H

#include <memory>
#include <utility>
#include <vector>

#include "devtypes.H"
#include "geom.H"
#include "hostmem.H"

namespace cmg {

enum { CHUNK = 256 };

// Allocator whose resize leaves new elements uninitialised: the largest
// plan tables (coarse-fine stencils, flux registers) are resized once and
// filled by their builders on host threads, so each page is first touched by
// the thread that writes it instead of by one thread zeroing them all.  Their
// storage comes from the kept large blocks (hostBlockAlloc), so plans built
// after others were freed reuse mapped pages.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  T* allocate(size_t n) { return static_cast<T*>(hostBlockAlloc(n * sizeof(T))); }
  void deallocate(T* p, size_t n) { hostBlockFree(p, n * sizeof(T)); }
  template <class U>
  NoInitAlloc(const NoInitAlloc<U>&) {}
  template <class U>
  void construct(U* p) noexcept {
    ::new ((void*)p) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new ((void*)p) U(std::forward<A>(a)...);
  }
};
template <class T>
using PlanVec = std::vector<T, NoInitAlloc<T>>;

struct LevelPlan {
  Layout grids;
  BoxIndex index;  // spatial index of grids
  Box domain;
  double dx = 0, dxCrse = 0;   // dxCrse: spacing of the coarser AMR level (2 dx)
  std::vector<BoxDesc> boxes;
  int64_t nelem = 0;           // elements per field on this level
  // Ghost work: [0, nExchBC) exchange + physical BC, then homogeneous CF.
  std::vector<GhostTask> ghost;
  int nExchBC = 0;
  // Cumulative cell counts of the ghost tasks (ghostStart[t] = first cell of
  // task t), so one ghost kernel can spread cells evenly over thread blocks.
  std::vector<int> ghostStart;
  std::vector<int> ghostBlock;         // task holding cell b*GHOST_PER_BLOCK
  // The same over one-colour slots (colourSlots per task).
  std::vector<int> slotStart, slotBlock;
  // The ghost fill cell by cell: [colour 0 exchange+BC | colour 0 CF |
  // colour 1 exchange+BC | colour 1 CF], each group in task order.
  PlanVec<GhostCell> gcells;
  int gcStart[2] = {0, 0}, gcExch[2] = {0, 0}, gcCF[2] = {0, 0};
  // Face-ghost rules for relaxation without ghost fills: per box, six faces
  // (direction-major, low side first), each over its two tangential
  // directions in increasing order; faceOff[6*b + 2*d + (side > 0)].
  std::vector<FaceRule> faceRules;
  std::vector<int> faceOff;
  // Colour-1 cells on exchange faces (DeferredCell), box by box, x fastest;
  // empty until the fused sweep asks for them (buildDeferred).
  std::vector<DeferredCell> deferred;
  // Face ghosts read by each chunk of a colour pass (chunksColor[c]): the
  // fill entries of chunk q are chunkGhost[c][chunkGhostStart[c][q] ..
  // chunkGhostStart[c][q + 1]).
  std::vector<GhostCell> chunkGhost[2];
  std::vector<int> chunkGhostStart[2];
  std::vector<GhostTask> zeroCovered;  // covered by the next finer level
  std::vector<int> zeroStart;          // cumulative cell counts of zeroCovered
  std::vector<int> zeroBlock;
  std::vector<Chunk> chunksAll, chunksColor[2];
  // Coarse-fine interpolation from the next coarser level (levels >= 1).
  PlanVec<CFCoarse> cfCoarse;
  PlanVec<CFFine> cfFine;
  PlanVec<double> cfW;
  PlanVec<int64_t> cfOff;
  // Maps to the next coarser level (levels >= 1): items in coarse index space.
  std::vector<CoarseFineItem> toCoarse;
  std::vector<Chunk> toCoarseChunksF;  // chunks over fine cells of items
  std::vector<Chunk> toCoarseChunksC;  // chunks over coarse cells of items
  // Flux-register correction of this level from the next finer level.
  PlanVec<RefluxCell> rfCells;
  PlanVec<RefluxCoarseTerm> rfCoarse;
  PlanVec<RefluxFineGroup> rfFine;
  // Forest levels (mergeLevels): hierarchy of each box, first element of each
  // hierarchy (one more entry: nelem).  Empty for one hierarchy.
  std::vector<int> boxHier;
  std::vector<int64_t> hierStart;
};

// Compact indexing of the bottom level for the bottom solve: valid cells
// first (box by box, x fastest, the reference's summation order), then the
// face-ghost slots the 7-point stencil reads (where the face coefficients of
// a variable-coefficient operator are gathered).  The solve's vectors hold
// the valid slots; a ghost's value is read from its source through nbv.
struct BottomPlan {
  int nv = 0, ng = 0;            // valid cells, ghost slots
  std::vector<int> fab;          // FAB element index of every slot (nv + ng)
  std::vector<int> nb;           // 6 neighbour slots per valid cell (+x,-x,+y,-y,+z,-z)
  std::vector<int> color[2];     // valid slots of each colour
  std::vector<int> boxStart;     // first valid slot of each box (nbox + 1)
  std::vector<int> gsrc, gkind;  // per ghost slot: source slot, 0 copy / 1 Dirichlet / 2 untouched
  std::vector<int> nbv;          // 6 per valid cell: the neighbour's value source, a valid slot s
                                 // (read as is) or -(s + 1) (a Dirichlet ghost: 0 - value)
};
void buildBottom(const LevelPlan& L, BottomPlan& B);

// Face-ghost rules of a level from its ghost tasks (LevelPlan::faceRules).
void buildFaceRules(LevelPlan& L);
// buildFaceRules unless the level has them; true when it built them.
bool ensureFaceRules(LevelPlan& L);
// The per-chunk face-ghost lists of the prefill relaxation variant
// (LevelPlan::chunkGhost, and the face rules they are made from) on levels of
// at most kPrefillMaxCells cells that lack them; true when it built them.
bool ensureChunkGhosts(LevelPlan& L);
// The colour-1 cells on exchange faces (LevelPlan::deferred), for the fused
// sweep; built on demand, after the face rules.
void buildDeferred(LevelPlan& L);
// Levels of at most this many cells get the per-chunk ghost lists of the
// prefill relaxation variant (LevelPlan::chunkGhost).
constexpr int64_t kPrefillMaxCells = int64_t(1) << 22;
// Levels up to this many cells get their face rules with the plan (the
// one-block relaxation uses them); larger ones only when the fused sweep asks
// for them (ensureFaceRules).
constexpr int64_t kFaceRulesEagerCells = 32768;

// Layout and ghost/chunk plans of one level (AMR level or multigrid depth).
// dxCrse > 0 enables homogeneous coarse-fine ghost tasks on CF faces.
// bc: homogeneous boundary type of each domain face (x-lo, x-hi, y-lo, y-hi,
// z-lo, z-hi): 0 Dirichlet, 1 Neumann; nullptr for Dirichlet everywhere.
// periodic: per direction, the domain repeats (exchange from its images, no
// boundary values); nullptr for none.
void buildLevel(LevelPlan& L, const Layout& grids, const Box& domain, double dx, double dxCrse,
                const int* bc = nullptr, const bool* periodic = nullptr);
// Coarse-fine interpolation tables of fine level F from coarse level C.
void buildQuadCF(LevelPlan& F, const LevelPlan& C);
// Coarse/fine box maps and zero-covered tasks (F fine, C coarse).
void buildCoarseFine(LevelPlan& F, LevelPlan& C);
// Flux-register lists for coarse level C with finer level F.  vc selects the
// variable-coefficient flux (face coefficients are then addressed).
void buildReflux(LevelPlan& C, const LevelPlan& F, bool vc);

// Cell index of (i,j,k) inside box b of level L.
inline int64_t cellOf(const LevelPlan& L, int b, const IV& p) {
  return cellIndex(L.boxes[b], p[0], p[1], p[2]);
}

// blockTask[b] = task holding cell b*GHOST_PER_BLOCK for cumulative cell
// counts `start` (one entry per block plus a last one = last task).
std::vector<int> blockTasks(const std::vector<int>& start);

// Finds the box of L containing p, or -1.
int ownerOf(const LevelPlan& L, const IV& p);

// The same level of several hierarchies as one level (a forest level):
// parts[k] placed at element offset elemOff[k] and box offset boxOff[k];
// coarseElemOff / coarseBoxOff (the next coarser level's part offsets) shift
// the coarse-fine tables, fineElemOff (the next finer level's) the flux
// register; nullptr where the level has no such neighbour.
void mergeLevels(const std::vector<const LevelPlan*>& parts, const std::vector<int64_t>& elemOff,
                 const std::vector<int>& boxOff, const std::vector<int64_t>* coarseElemOff,
                 const std::vector<int>* coarseBoxOff, const std::vector<int64_t>* fineElemOff, LevelPlan& out);

}  // namespace cmg

#endif
