// Coarse-to-fine interpolation of a new fine level (AMRTools/FineInterp.cpp:
// FineInterp::interpToFine with the default PCInterp boundary limit type, and
// pwcinterpToFine), refinement ratio 2, one component.
//
// The reference copies the coarse level into the coarsened fine layout with
// one ghost layer (FineInterp.cpp:148-160), then per fine box fills every fine
// cell with its coarse parent (interpconstant) and, on b_mod = the coarsened
// box trimmed one cell from the domain boundary (FineInterp.cpp:285-292),
// adds the limited central slopes (interpcentralslope, interplimit,
// interplinear; InterpF.ChF).  Here a thread block per fine box loads
// grow(coarsen(fine box), 1) & domain from the coarse level into shared
// memory, and one thread per coarse cell computes the three slopes and the
// limiter from it and writes the eight fine cells with the reference's
// operations in its order (boxes whose staging block exceeds shared memory
// take a gather kernel into device memory and a second kernel).  Slopes on the domain-boundary layer
// (interphisideslope / interplosideslope) feed nothing: those cells stay
// piecewise constant, as in the reference.
#ifndef CMG_FINEINTERP_H
#define CMG_FINEINTERP_H

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "devtypes.H"
#include "geom.H"

namespace cmg {

// One fine box: its coarsened box b, b_mod (empty when some mhi < mlo) and
// its staging block (b grown by one, x fastest).
struct FiBox {
  int fbox;
  int lo[3], hi[3];
  int mlo[3], mhi[3];
  int sx, sy;
  int gcells;    // cells of grow(b, 1) & domain that the coarse level holds
  int64_t soff;
};

// Cells of grow(b, 1) & domain that coarse box cbox holds (coarse index space).
struct FiGather {
  int fi, cbox;
  int lo[3], hi[3];
  int cstart;    // cells of the box's earlier items
};

// A box of a flat valid-cell array: cells x fastest from off.
struct FlatBox {
  int lo[3];
  int nx, ny;
  int64_t off;
};

// Flat valid-cell tables of a layout (the C ABI's order); returns the cells.
int64_t flatBoxes(const std::vector<Box>& grids, std::vector<FlatBox>& out);

class FineInterpOp {
 public:
  // coarse: the coarse layout with its spatial index; coarseDomain: the
  // coarse problem domain; fine: the fine layout (boxes coarsenable by 2).
  // allowFused = false keeps the two-kernel path whatever the box sizes.
  FineInterpOp(const std::vector<Box>& coarse, const BoxIndex& cindex, const Box& coarseDomain,
               const std::vector<Box>& fine, cudaStream_t s, bool allowFused = true);
  ~FineInterpOp();
  FineInterpOp(const FineInterpOp&) = delete;
  FineInterpOp& operator=(const FineInterpOp&) = delete;
  // grow(coarsen(fine box), 1) & domain lies in the coarse layout for every
  // fine box (what the limited interpolation reads); coarsen(fine box) does
  // (what the piecewise-constant one reads).
  bool nested() const { return nested_; }
  bool covered() const { return covered_; }
  // Red-black level fields (BoxDesc tables of the two levels).
  void run(const BoxDesc* cboxes, const double* coarse, const BoxDesc* fboxes, double* fine, bool pwc);
  // Flat valid-cell arrays (FlatBox tables of the two levels, on the device).
  void runFlat(const FlatBox* cboxes, const double* coarse, const FlatBox* fboxes, double* fine, bool pwc);
  int64_t fineCells() const { return fineCells_; }
  // one kernel with the staging blocks in shared memory (every block fits)
  bool fused() const { return fused_; }
  // Stream the interpolation kernels run on from now on (the plan's memory
  // stays with the stream given at construction, which must outlive this).
  void setStream(cudaStream_t s) { s_ = s; }

 private:
  void check(bool pwc) const;
  cudaStream_t s_, own_;
  bool nested_ = true, covered_ = true;
  int64_t fineCells_ = 0, stageCells_ = 0;
  int nBoxCh_ = 0, nGatherCh_ = 0, nbox_ = 0;
  bool fused_ = false;
  size_t smem_ = 0;
  void* mem_ = nullptr;  // one allocation: boxes, chunks, gathers, staging
  const FiBox* boxes_ = nullptr;
  const Chunk* boxCh_ = nullptr;
  const FiGather* gathers_ = nullptr;
  const Chunk* gatherCh_ = nullptr;
  const int* itemStart_ = nullptr;  // gather items of each fine box (nbox + 1)
  double* stage_ = nullptr;
};

}  // namespace cmg

#endif
