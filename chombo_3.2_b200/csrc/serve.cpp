// Request loop (see serve.H).
#include "serve.H"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <functional>
#include <map>
#include <cstdio>

#include "meshrefine.H"
#include "synthfill.H"
#include "tagging.H"

namespace cmg {

namespace {

using Clock = std::chrono::steady_clock;

// FNV-1a over the 64-bit words of the values.
uint64_t fnv1a(const double* v, size_t n, uint64_t h) {
  for (size_t i = 0; i < n; ++i) {
    uint64_t w;
    std::memcpy(&w, &v[i], sizeof(w));
    h ^= w;
    h *= 1099511628211ULL;
  }
  return h;
}

int64_t fabElements(const Box& b) {
  const int64_t px = (b.size(0) + 3) & ~1;
  return px * (b.size(1) + 2) * (b.size(2) + 2);
}

}  // namespace

size_t estimateDeviceBytes(const std::vector<std::vector<Box>>& boxes, bool vc, bool mixed) {
  // Per AMR level: 6 FP64 fields (+5 coefficient arrays), FP32 copies of 4
  // fields (+5) for mixed precision; multigrid depths below level 0 add at
  // most 1/7 of level 0; plans and ghost lists about 30% more.
  const double f64 = 6 + (vc ? 5 : 0), f32 = mixed ? 4 + (vc ? 5 : 0) : 0;
  double bytes = 0;
  for (size_t l = 0; l < boxes.size(); ++l) {
    int64_t n = 0;
    for (const Box& b : boxes[l]) n += fabElements(b);
    double lev = n * (8.0 * f64 + 4.0 * f32);
    bytes += l == 0 ? lev * (1.0 + 1.0 / 7.0) : lev;
  }
  return (size_t)(bytes * 1.3) + (64u << 20);
}

namespace {

// Failure of one request: its status and message.
struct RequestError : std::runtime_error {
  int code;
  RequestError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// The description checks the C ABI used to apply to the whole call, now per
// request (an invalid request fails alone).
void validate(const Request& q) {
  auto bad = [](const char* what) { throw RequestError(REQ_EINVAL, std::string("cmg: invalid request: ") + what); };
  if (q.n0 < 8) bad("base size below 8");
  if (q.levels < 1) bad("no levels");
  if (q.op != 0 && q.op != 1) bad("operator is 0 (AMRPoissonOp) or 1 (VCAMRPoissonOp2)");
  if (q.blockFactor < 1 || q.maxBox < 0) bad("blocking factor or maximum box size");
  if (q.maxBox > 0 && q.maxBox % q.blockFactor != 0) bad("maximum box size not a multiple of the blocking factor");
  if (q.n0 % q.blockFactor != 0) bad("base size not a multiple of the blocking factor");
  const SolveParams& p = q.params;
  if (p.pre < 0 || p.post < 0 || p.bottom < 0 || p.numMG < 1 || p.iterMax < 0) bad("solver parameters");
  if (!(p.eps > 0) || !(q.timeout >= 0)) bad("tolerance or time limit");
}

// What requests must share to be solved as one forest: the problem recipe
// (so the same level-0 layout and multigrid depths), operator, precision and
// every solver parameter but the tolerance (each member keeps its own).
std::string classKey(const Request& q) {
  const SolveParams& p = q.params;
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%d %d %d %d %.17g %.17g %d %.17g %.17g %d %d %d %d %d %d %d %d %.17g %.17g %d",
                q.n0, q.levels, q.maxBox, q.blockFactor, q.fillRatio, q.thresh, q.op, q.alpha, q.beta, (int)q.mixed,
                (int)q.graphs, p.pre, p.post, p.bottom, p.numMG, p.iterMax, p.imin, p.hang, p.normThresh, p.iterMin);
  return buf;
}

// Requests waiting to be solved together (ServeOptions::batchWindow).
struct Batch {
  std::vector<size_t> members;                  // request indices, the first is the leader
  std::vector<std::vector<std::vector<Box>>> boxes;
  std::vector<Clock::time_point> starts;        // when each member's own processing began
  Clock::time_point deadline;
  bool closed = false, done = false;
};

}  // namespace

double serve(const std::vector<Request>& reqs, const ServeOptions& opt, std::vector<RequestResult>& out) {
  const size_t n = reqs.size();
  out.assign(n, RequestResult());
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return reqs[a].arrival < reqs[b].arrival; });
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cmg: no CUDA device");

  std::mutex m;
  std::condition_variable cv;
  size_t next = 0;
  double used = 0;
  const Clock::time_point t0 = Clock::now();
  auto since = [&](Clock::time_point t) { return std::chrono::duration<double>(t - t0).count(); };
  auto at = [&](double sec) { return t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(sec)); };
  // Why request q must stop now (0: it may go on).
  auto stopFor = [&](const Request& q) -> int {
    if (q.cancel && *q.cancel) return REQ_ECANCELLED;
    if (q.timeout > 0 && Clock::now() >= at((opt.openLoop ? q.arrival : 0.0) + q.timeout)) return REQ_ETIMEOUT;
    return REQ_OK;
  };
  auto stopMessage = [](int code) {
    return std::string(code == REQ_ECANCELLED ? "cmg: request cancelled" : "cmg: request time limit passed");
  };
  std::mutex bm;
  std::condition_variable bcv;
  std::map<std::string, std::shared_ptr<Batch>> openBatches;

  // One forest for the members of a batch, on the leader's stream: every
  // member's result (or error) is written here.
  auto runBatch = [&](Batch& b, cudaStream_t s) {
    const size_t K = b.members.size();
    const Request& q0 = reqs[b.members[0]];
    try {
      std::vector<HierarchyDesc> descs(K);
      for (size_t k = 0; k < K; ++k) {
        const Request& q = reqs[b.members[k]];
        HierarchyDesc& d = descs[k];
        d.domain = Box(IV(0, 0, 0), IV(q.n0 - 1, q.n0 - 1, q.n0 - 1));
        d.dx0 = 1.0 / q.n0;
        d.boxes = b.boxes[k];
        d.vc = q.op;
        d.alpha = q.alpha;
        d.beta = q.beta;
      }
      const Clock::time_point tb = Clock::now();
      std::unique_ptr<Solver> S(new Solver(descs, s));
      const Clock::time_point tf = Clock::now();
      std::vector<uint64_t> seeds;
      for (size_t k = 0; k < K; ++k) seeds.push_back(reqs[b.members[k]].seed);
      S->fillSyntheticForest(seeds);
      const int fl = S->numLevels() - 1;
      int box0 = 0;
      for (size_t k = 0; k < K; ++k) {
        if (reqs[b.members[k]].injectNanRHS) {
          // one valid cell of member k's finest right-hand side made NaN
          const BoxDesc& bd = S->level(fl).boxes[box0];
          const double nan = std::nan("");
          if (cudaMemcpy(S->devRHS(fl) + cellIndex(bd, bd.lo[0], bd.lo[1], bd.lo[2]), &nan, sizeof(double),
                         cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("cmg: fault injection copy");
        }
        box0 += (int)b.boxes[k][fl].size();
      }
      S->setUseGraphs(q0.graphs);
      S->setRelaxMode(1);  // one solve per hierarchy: no autotuning (see below)
      const Clock::time_point tsolve = Clock::now();
      std::vector<double> eps;
      std::vector<std::function<int(int)>> ints;
      for (size_t k = 0; k < K; ++k) {
        const Request* q = &reqs[b.members[k]];
        eps.push_back(q->params.eps);
        ints.push_back([q, &stopFor](int iter) -> int {
          if (q->injectCancelAfter >= 0 && iter >= q->injectCancelAfter) return REQ_ECANCELLED;
          return stopFor(*q);
        });
      }
      const std::vector<SolveResult> res = S->solveForest(q0.params, true, q0.mixed, &eps, &ints);
      const Clock::time_point tsolved = Clock::now();
      std::vector<uint64_t> hash(K, 1469598103934665603ULL);
      std::vector<int64_t> cells(K, 0);
      std::vector<double> phi;
      for (int l = 0; l < S->numLevels(); ++l) {
        phi.resize(S->numValidCells(l));
        S->getPhi(l, phi.data(), false);
        size_t at0 = 0;
        for (size_t k = 0; k < K; ++k) {
          const int64_t nk = S->hierarchyCells((int)k, l);
          hash[k] = fnv1a(phi.data() + at0, (size_t)nk, hash[k]);
          cells[k] += nk;
          at0 += (size_t)nk;
        }
      }
      const size_t bytes = S->deviceBytes();
      for (size_t k = 0; k < K; ++k) {
        RequestResult& r = out[b.members[k]];
        r.batchSize = (int)K;
        r.buildSeconds = std::chrono::duration<double>(tf - tb).count();
        r.fillSeconds = std::chrono::duration<double>(tsolve - tf).count();
        r.setupSeconds = std::chrono::duration<double>(tsolve - b.starts[k]).count();
        r.started = since(tsolve);
        r.solved = since(tsolved);
        r.solveSeconds = std::chrono::duration<double>(tsolved - tsolve).count();
        r.exitStatus = res[k].exitStatus;
        r.iterations = res[k].iterations;
        r.r0 = res[k].history.front();
        r.rfinal = res[k].history.back();
        r.cells = cells[k];
        r.deviceBytes = bytes / K;
        if (res[k].interrupted) {
          r.error = res[k].interrupted;
          r.message = stopMessage(res[k].interrupted);
        } else if (res[k].diverged) {
          r.error = REQ_EDIVERGED;
          r.message = "cmg: residual norm is not finite after " + std::to_string(res[k].iterations) + " iterations";
        } else {
          r.phiHash = hash[k];
        }
      }
      cudaStreamSynchronize(s);
    } catch (...) {
      std::string w = "cmg: unknown error";
      try {
        throw;
      } catch (const std::exception& e) {
        w = e.what();
      } catch (...) {
      }
      for (size_t k = 0; k < K; ++k) {
        RequestResult& r = out[b.members[k]];
        r.batchSize = (int)K;
        r.error = w.find("cudaMalloc") != std::string::npos ? REQ_ENOMEM : REQ_EINTERNAL;
        r.message = w;
      }
    }
  };

  auto work = [&]() {
    cudaSetDevice(dev);
    for (;;) {
      size_t idx;
      {
        std::lock_guard<std::mutex> lk(m);
        if (next >= n) return;
        idx = order[next++];
      }
      const Request& q = reqs[idx];
      RequestResult& r = out[idx];
      if (opt.openLoop) std::this_thread::sleep_until(at(q.arrival));
      const bool limited = q.timeout > 0;
      const Clock::time_point deadline = at((opt.openLoop ? q.arrival : 0.0) + q.timeout);
      // Why the request must stop now (0: it may go on).
      auto stopCode = [&]() -> int {
        if (q.cancel && *q.cancel) return REQ_ECANCELLED;
        if (limited && Clock::now() >= deadline) return REQ_ETIMEOUT;
        return REQ_OK;
      };
      auto stopError = [&](int code) {
        throw RequestError(code, code == REQ_ECANCELLED ? "cmg: request cancelled" : "cmg: request time limit passed");
      };
      double est = 0;
      bool reserved = false;
      cudaStream_t s = nullptr;
      try {
        validate(q);
        if (int c = stopCode()) stopError(c);
        const Clock::time_point ts = Clock::now();
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
          throw std::runtime_error("cmg: stream");
        std::vector<std::vector<Box>> boxes;
        if (q.deviceTags) {
          DeviceTagger tagger(s);
          boxes = syntheticHierarchy(q.n0, q.levels, q.maxBox, q.blockFactor, q.fillRatio, q.seed, q.thresh, &tagger);
        } else {
          boxes = syntheticHierarchy(q.n0, q.levels, q.maxBox, q.blockFactor, q.fillRatio, q.seed, q.thresh);
        }
        r.gridSeconds = std::chrono::duration<double>(Clock::now() - ts).count();
        est = (double)estimateDeviceBytes(boxes, q.op == 1, q.mixed);
        r.estimate = (size_t)est;
        if (est > opt.hbmBudget)
          throw RequestError(REQ_ENOMEM, "cmg: request needs about " + std::to_string((long long)est) +
                                             " device bytes, more than the whole budget of " +
                                             std::to_string((long long)opt.hbmBudget));
        {
          // Admission: wait until the request fits beside the admitted ones,
          // looking at cancellation and the time limit every 5 ms.
          std::unique_lock<std::mutex> lk(m);
          while (!(used + est <= opt.hbmBudget)) {
            if (int c = stopCode()) {
              lk.unlock();
              stopError(c);
            }
            cv.wait_for(lk, std::chrono::milliseconds(5));
          }
          used += est;
          reserved = true;
        }
        r.admitted = since(Clock::now());
        bool batched = false;
        if (opt.batchWindow > 0 && opt.maxBatch > 1) {
          // Join the open batch of this request's class, or open one and lead it.
          const std::string key = classKey(q);
          std::shared_ptr<Batch> b;
          bool leader = false;
          {
            std::unique_lock<std::mutex> lk(bm);
            auto it = openBatches.find(key);
            if (it != openBatches.end() && !it->second->closed) {
              b = it->second;
              b->members.push_back(idx);
              b->boxes.push_back(boxes);
              b->starts.push_back(ts);
              if ((int)b->members.size() >= opt.maxBatch) {
                b->closed = true;
                openBatches.erase(it);
              }
              bcv.notify_all();
            } else {
              b = std::make_shared<Batch>();
              b->members.push_back(idx);
              b->boxes.push_back(boxes);
              b->starts.push_back(ts);
              b->deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                               std::chrono::duration<double>(opt.batchWindow));
              openBatches[key] = b;
              leader = true;
              while (!b->closed && Clock::now() < b->deadline) bcv.wait_until(lk, b->deadline);
              if (!b->closed) {
                b->closed = true;
                auto it2 = openBatches.find(key);
                if (it2 != openBatches.end() && it2->second == b) openBatches.erase(it2);
              }
            }
            if (!leader) {
              while (!b->done) bcv.wait(lk);
              batched = true;
            }
          }
          if (leader && b->members.size() > 1) {
            runBatch(*b, s);
            {
              std::lock_guard<std::mutex> lk(bm);
              b->done = true;
            }
            bcv.notify_all();
            batched = true;
          }
          if (batched && r.error) throw RequestError(r.error, r.message);
        }
        if (!batched) {
        HierarchyDesc d;
        d.domain = Box(IV(0, 0, 0), IV(q.n0 - 1, q.n0 - 1, q.n0 - 1));
        d.dx0 = 1.0 / q.n0;
        d.boxes = boxes;
        d.vc = q.op;
        d.alpha = q.alpha;
        d.beta = q.beta;
        {
          const Clock::time_point tb = Clock::now();
          std::unique_ptr<Solver> S(new Solver(d, s));
          const Clock::time_point tf = Clock::now();
          r.buildSeconds = std::chrono::duration<double>(tf - tb).count();
          S->fillSyntheticDevice(q.seed);
          if (q.injectNanRHS) {
            // one valid cell of the finest right-hand side made NaN
            const int fl = S->numLevels() - 1;
            const BoxDesc& b0 = S->level(fl).boxes[0];
            const double nan = std::nan("");
            if (cudaMemcpy(S->devRHS(fl) + cellIndex(b0, b0.lo[0], b0.lo[1], b0.lo[2]), &nan, sizeof(double),
                           cudaMemcpyHostToDevice) != cudaSuccess)
              throw std::runtime_error("cmg: fault injection copy");
          }
          r.fillSeconds = std::chrono::duration<double>(Clock::now() - tf).count();
          S->setUseGraphs(q.graphs);
          // A served hierarchy is solved once: the relaxation autotuner's
          // timing sweeps (and the per-chunk lists it would build) cost more
          // than the variants it can pick save, so every level keeps the
          // ghost-fill variant.
          S->setRelaxMode(1);
          const Clock::time_point tsolve = Clock::now();
          r.setupSeconds = std::chrono::duration<double>(tsolve - ts).count();
          r.started = since(tsolve);
          SolveParams sp = q.params;
          sp.interrupt = [&](int iter) -> int {
            if (q.injectCancelAfter >= 0 && iter >= q.injectCancelAfter) return REQ_ECANCELLED;
            return stopCode();
          };
          SolveResult res = q.mixed ? S->solveMixed(sp) : S->solve(sp);
          const Clock::time_point tsolved = Clock::now();
          r.solveSeconds = std::chrono::duration<double>(tsolved - tsolve).count();
          r.solved = since(tsolved);
          r.exitStatus = res.exitStatus;
          r.iterations = res.iterations;
          r.r0 = res.history.front();
          r.rfinal = res.history.back();
          if (res.interrupted) stopError(res.interrupted);
          if (res.diverged)
            throw RequestError(REQ_EDIVERGED, "cmg: residual norm is not finite after " +
                                                  std::to_string(res.iterations) + " iterations");
          uint64_t h = 1469598103934665603ULL;
          std::vector<double> phi;
          for (int l = 0; l < S->numLevels(); ++l) {
            phi.resize(S->numValidCells(l));
            S->getPhi(l, phi.data(), false);
            h = fnv1a(phi.data(), phi.size(), h);
            r.cells += S->numValidCells(l);
          }
          r.phiHash = h;
          r.deviceBytes = S->deviceBytes();
        }
        }  // the request alone
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        s = nullptr;
      } catch (const RequestError& e) {
        r.error = e.code;
        r.message = e.what();
      } catch (const std::bad_alloc& e) {
        r.error = REQ_ENOMEM;
        r.message = e.what();
      } catch (const std::exception& e) {
        const std::string w = e.what();
        r.error = w.find("cudaMalloc") != std::string::npos ? REQ_ENOMEM : REQ_EINTERNAL;
        r.message = w;
      } catch (...) {
        r.error = REQ_EINTERNAL;
        r.message = "cmg: unknown error";
      }
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
      r.finished = since(Clock::now());
      if (reserved) {
        std::lock_guard<std::mutex> lk(m);
        used -= est;
      }
      cv.notify_all();
    }
  };
  const int nw = std::max(1, std::min<int>(opt.maxInflight, (int)std::max<size_t>(n, 1)));
  std::vector<std::thread> th;
  for (int w = 0; w < nw; ++w) th.emplace_back(work);
  for (auto& t : th) t.join();
  return since(Clock::now());
}

}  // namespace cmg
