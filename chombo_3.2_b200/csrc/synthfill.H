// Seeded synthetic inputs of the benchmark workloads on a hierarchy: the
// Gaussian-bump right-hand side at cell centres of every level and, for the
// variable-coefficient operator, a(x) at cell centres and b(x) at face
// centres (exp of a seeded Fourier series, in [0.1, 10]), then the
// coefficient finalisation.  Same values as the oracle driver's.
#ifndef CMG_SYNTHFILL_H
#define CMG_SYNTHFILL_H

#include <cstdint>

#include "solver.H"

namespace cmg {

void fillSynthetic(Solver& S, bool vc, uint64_t seed);

}  // namespace cmg

#endif
