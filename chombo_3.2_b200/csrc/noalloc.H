// Limits of the allocation-free residual norm (noalloc.cu).
#ifndef CMG_NOALLOC_H
#define CMG_NOALLOC_H

namespace cmg {

class Solver;

// Static scratch: one FP64 partial per box of a level plus one running
// maximum, (4096 + 1) * 8 bytes per device.
enum { NOALLOC_MAX_BOXES = 4096, NOALLOC_MAX_LEVELS = 16, NOALLOC_MAX_DEVICES = 64 };

// Composite residual max-norm of the hierarchy's current phi and rhs, same
// value as Solver::residualNorm, allocating no memory on success.
double residualNormNoAlloc(Solver& S);
// Drops the scratch addresses found so far (after a device reset).
void forgetNoAllocScratch();

}  // namespace cmg

#endif
