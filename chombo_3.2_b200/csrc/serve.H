// Request loop for many independent solves on one GPU (batching and
// serving; no counterpart in the reference, which solves one hierarchy per
// call).  Each request describes a seeded synthetic problem: the example
// hierarchy (grid generation of meshrefine.H), Poisson/Helmholtz or the
// variable-coefficient operator, a tolerance and the precision.  Workers
// admit requests in arrival order as long as the device memory held by the
// admitted hierarchies stays within a budget, build each hierarchy (plans,
// device state, inputs) on its own CUDA stream, solve it (CUDA-graph replay
// of each iteration), read phi back and release the memory, so that the
// solves of all in-flight requests overlap on the device.  Requests never
// share device data, so each result is the same alone and in the mix.
#ifndef CMG_SERVE_H
#define CMG_SERVE_H

#include <cstdint>
#include <string>
#include <vector>

#include "solver.H"

namespace cmg {

struct Request {
  double arrival = 0;  // seconds after the start of the run (open loop)
  int n0 = 32, levels = 1, maxBox = 32, blockFactor = 8;
  double fillRatio = 0.75, thresh = 0.1;
  uint64_t seed = 20261203;
  int op = 0;  // 0: AMRPoissonOp, 1: VCAMRPoissonOp2
  double alpha = 0.0, beta = 1.0;
  SolveParams params;
  bool mixed = true, graphs = true;
  bool deviceTags = false;  // tagging pass of the grid generation on the device (tagging.H)
  double timeout = 0;       // seconds after arrival to finish by (0: no limit)
  const volatile int* cancel = nullptr;  // set non-zero by the caller (any thread) to cancel
  // Host-side fault injection for tests: a NaN in the right-hand side of the
  // finest level after the inputs are generated; cancellation after this
  // many iterations (-1: never).
  bool injectNanRHS = false;
  int injectCancelAfter = -1;
};

struct RequestResult {
  int exitStatus = -1, iterations = 0;
  double admitted = 0, started = 0, solved = 0, finished = 0;  // seconds after the start
  double setupSeconds = 0, solveSeconds = 0;
  double gridSeconds = 0, buildSeconds = 0, fillSeconds = 0;  // parts of setupSeconds
  double r0 = 0, rfinal = 0;
  int64_t cells = 0;
  size_t deviceBytes = 0;
  uint64_t phiHash = 0;  // FNV-1a over the 64-bit words of phi on every level (valid cells)
  size_t estimate = 0;   // admission estimate of the device bytes
  int batchSize = 1;     // requests solved together with this one (one forest), itself included
  int error = 0;         // 0 or a CMG_* status (cmg.h)
  std::string message;   // what went wrong when error != 0
};

struct ServeOptions {
  double hbmBudget = 120e9;  // bytes of device memory the admitted hierarchies may hold
  int maxInflight = 16;      // worker threads, each owning one hierarchy at a time
  bool openLoop = true;      // release requests at their arrival times
  // Batching V-cycles across requests: a request of the same class as one
  // admitted less than batchWindow seconds earlier (same problem recipe,
  // operator, precision and solver parameters but the tolerance) joins it,
  // and up to maxBatch of them are solved as one forest (Solver's forest
  // constructor: one launch per V-cycle operation for all of them, each with
  // its own tolerance, stopping rule, time limit and cancellation).  0: every
  // request alone.
  double batchWindow = 0;
  int maxBatch = 16;
};

// Status codes of a request (the C ABI's CMG_* values).
enum { REQ_OK = 0, REQ_EINVAL = 1, REQ_ENOMEM = 2, REQ_ECUDA = 3, REQ_EINTERNAL = 4, REQ_EDIVERGED = 5,
       REQ_ETIMEOUT = 6, REQ_ECANCELLED = 7 };

// Runs every request; returns the wall time of the run in seconds.  A
// request that fails (invalid description, more memory than the whole
// budget, a non-finite residual, its time limit, cancellation, an error
// while it runs) gets its status and message and releases what it held; the
// other requests are not affected.
double serve(const std::vector<Request>& reqs, const ServeOptions& opt, std::vector<RequestResult>& out);

// Device bytes a request's hierarchy will hold, from its box lists (the
// admission estimate; the real figure is recorded after creation).
size_t estimateDeviceBytes(const std::vector<std::vector<Box>>& boxes, bool vc, bool mixed);

}  // namespace cmg

#endif
