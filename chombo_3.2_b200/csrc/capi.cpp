// C ABI over the solver (include/cmg.h).  Every entry point catches
// exceptions and turns them into status codes; nothing aborts.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cmg.h"
#include "hostmem.H"
#include "hostpool.H"
#include "fineinterp.H"
#include "meshrefine.H"
#include "noalloc.H"
#include "serve.H"
#include "solver.H"
#include "synthfill.H"
#include "tagging.H"

struct cmg_hierarchy {
  cudaStream_t stream = nullptr;
  cmg::Solver* solver = nullptr;
  cmg::HierarchyDesc desc;
};

struct cmg_fine_interp {
  cudaStream_t stream = nullptr;  // own stream: plan memory, and the work until cmg_fine_interp_set_stream
  cudaStream_t work = nullptr;    // stream of the interpolation work
  cmg::FineInterpOp* op = nullptr;
  int64_t ncoarse = 0, nfine = 0;
  void* mem = nullptr;  // FlatBox tables of both layouts, then coarse and fine staging for host data
  const cmg::FlatBox* cflat = nullptr;
  const cmg::FlatBox* fflat = nullptr;
  double* dcoarse = nullptr;
  double* dfine = nullptr;
};

namespace {

thread_local std::string g_err;

// A solve whose residual norm became NaN or infinite: its outputs are
// written, and the call returns CMG_EDIVERGED.
struct Diverged : std::runtime_error {
  explicit Diverged(int iter)
      : std::runtime_error("cmg: residual norm is not finite after " + std::to_string(iter) + " iterations") {}
};

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

template <class F>
int guard(F fn) {
  try {
    fn();
    return CMG_OK;
  } catch (const Diverged& e) {
    return fail(CMG_EDIVERGED, e.what());
  } catch (const std::bad_alloc& e) {
    return fail(CMG_ENOMEM, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(CMG_EINVAL, e.what());
  } catch (const std::runtime_error& e) {
    std::string w = e.what();
    if (w.find("cudaMalloc") != std::string::npos) return fail(CMG_ENOMEM, w);
    if (w.find("cmg: ") == 0 && w.find(": ") != w.rfind(": ")) return fail(CMG_ECUDA, w);
    return fail(CMG_EINTERNAL, w);
  } catch (...) {
    return fail(CMG_EINTERNAL, "unknown error");
  }
}

void needLevel(const cmg_hierarchy* h, int level) {
  if (!h || !h->solver) throw std::invalid_argument("cmg: null hierarchy");
  if (level < 0 || level >= h->solver->numLevels()) throw std::invalid_argument("cmg: level out of range");
}

cmg::Box toBox(const cmg_box& b) { return cmg::Box(cmg::IV(b.lo[0], b.lo[1], b.lo[2]), cmg::IV(b.hi[0], b.hi[1], b.hi[2])); }

void fromBox(const cmg::Box& b, cmg_box& o) {
  for (int d = 0; d < 3; ++d) {
    o.lo[d] = b.lo[d];
    o.hi[d] = b.hi[d];
  }
}

void putMotion(int* o, int from, int to, const cmg::Box& fr, const cmg::Box& tr) {
  o[0] = from;
  o[1] = to;
  for (int d = 0; d < 3; ++d) {
    o[2 + d] = fr.lo[d];
    o[5 + d] = fr.hi[d];
    o[8 + d] = tr.lo[d];
    o[11 + d] = tr.hi[d];
  }
}

template <class F>
void parallelBoxes(size_t nbox, F fn) {
  hostParallel(nbox, [&](size_t b) { fn(b); });
}

}  // namespace

extern "C" {

const char* cmg_last_error(void) { return g_err.c_str(); }

int cmg_hierarchy_create(const int domain_lo[3], const int domain_hi[3], double dx0, int nlevels, const int* nboxes,
                         const cmg_box* boxes, int op, double alpha, double beta, cmg_hierarchy** out) {
  return cmg_hierarchy_create_bc(domain_lo, domain_hi, dx0, nlevels, nboxes, boxes, op, alpha, beta, nullptr, out);
}

namespace {
cmg::SolveParams solverParams(const cmg_solve_params* p);
}

// The checked description of one hierarchy (cmg_hierarchy_create_bc's
// arguments); boxes of nlevels levels, counts in nboxes.
static cmg::HierarchyDesc makeDesc(const int domain_lo[3], const int domain_hi[3], double dx0, int nlevels,
                                   const int* nboxes, const cmg_box* boxes, int op, double alpha, double beta,
                                   const int bc[6]) {
  if (!domain_lo || !domain_hi || !nboxes || !boxes || nlevels < 1 || dx0 <= 0 || (op != 0 && op != 1))
    throw std::invalid_argument("cmg: invalid hierarchy description");
  cmg::HierarchyDesc d;
  if (bc)
    for (int f = 0; f < 6; ++f) {
      if (bc[f] != CMG_BC_DIRICHLET && bc[f] != CMG_BC_NEUMANN && bc[f] != CMG_BC_PERIODIC)
        throw std::invalid_argument("cmg: boundary type is CMG_BC_DIRICHLET, CMG_BC_NEUMANN or CMG_BC_PERIODIC");
      if ((bc[f] == CMG_BC_PERIODIC) != (bc[f ^ 1] == CMG_BC_PERIODIC))
        throw std::invalid_argument("cmg: a periodic direction is periodic on both of its faces");
      d.bc[f] = bc[f] == CMG_BC_PERIODIC ? 0 : bc[f];
      d.periodic[f / 2] = bc[f] == CMG_BC_PERIODIC;
    }
  if (nlevels > 1 && (d.periodic[0] || d.periodic[1] || d.periodic[2]))
    throw std::invalid_argument("cmg: periodic domains are supported on one-level hierarchies");
  d.domain = cmg::Box(cmg::IV(domain_lo[0], domain_lo[1], domain_lo[2]), cmg::IV(domain_hi[0], domain_hi[1], domain_hi[2]));
  if (d.domain.empty()) throw std::invalid_argument("cmg: empty domain");
  d.dx0 = dx0;
  d.vc = op;
  d.alpha = alpha;
  d.beta = beta;
  int k = 0;
  cmg::Box dom = d.domain;
  for (int l = 0; l < nlevels; ++l) {
    if (nboxes[l] < 1) throw std::invalid_argument("cmg: a level has no boxes");
    if (l > 0) dom = dom.refine(2);
    std::vector<cmg::Box> v;
    for (int b = 0; b < nboxes[l]; ++b, ++k) {
      cmg::Box bx = toBox(boxes[k]);
      if (bx.empty() || !dom.contains(bx)) throw std::invalid_argument("cmg: box empty or outside its level domain");
      if (l > 0 && !bx.coarsenable(2)) throw std::invalid_argument("cmg: fine box not coarsenable by 2");
      v.push_back(bx);
    }
    std::vector<cmg::Box> sorted = v;
    std::sort(sorted.begin(), sorted.end());
    for (size_t i = 0; i < sorted.size(); ++i)
      for (size_t j = i + 1; j < sorted.size() && sorted[j].lo[0] <= sorted[i].hi[0]; ++j)
        if (sorted[i].intersects(sorted[j])) throw std::invalid_argument("cmg: boxes of a level overlap");
    d.boxes.push_back(v);
  }
  return d;
}

// A handle around a new Solver on its own stream.
static cmg_hierarchy* newHandle(const cmg::HierarchyDesc& d,
                                const std::function<cmg::Solver*(cudaStream_t)>& make) {
  cmg_hierarchy* h = new cmg_hierarchy;
  h->desc = d;
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    throw std::runtime_error(std::string("cmg: stream: ") + cudaGetErrorString(e));
  }
  try {
    h->solver = make(h->stream);
  } catch (...) {
    cudaStreamDestroy(h->stream);
    delete h;
    throw;
  }
  return h;
}

int cmg_hierarchy_create_bc(const int domain_lo[3], const int domain_hi[3], double dx0, int nlevels,
                            const int* nboxes, const cmg_box* boxes, int op, double alpha, double beta,
                            const int bc[6], cmg_hierarchy** out) {
  return guard([&]() {
    if (!out) throw std::invalid_argument("cmg: invalid hierarchy description");
    *out = nullptr;
    const cmg::HierarchyDesc d = makeDesc(domain_lo, domain_hi, dx0, nlevels, nboxes, boxes, op, alpha, beta, bc);
    *out = newHandle(d, [&](cudaStream_t s) { return new cmg::Solver(d, s); });
  });
}

int cmg_forest_create(int nh, const int domain_lo[3], const int domain_hi[3], double dx0, int nlevels,
                      const int* nboxes, const cmg_box* boxes, int op, double alpha, double beta, const int bc[6],
                      cmg_hierarchy** out) {
  return guard([&]() {
    if (!out || nh < 1 || nlevels < 1 || !nboxes || !boxes) throw std::invalid_argument("cmg: invalid forest");
    *out = nullptr;
    std::vector<cmg::HierarchyDesc> descs;
    size_t at = 0;
    for (int k = 0; k < nh; ++k) {
      descs.push_back(makeDesc(domain_lo, domain_hi, dx0, nlevels, nboxes + (size_t)k * nlevels, boxes + at, op,
                               alpha, beta, bc));
      for (int l = 0; l < nlevels; ++l) at += nboxes[(size_t)k * nlevels + l];
    }
    *out = newHandle(descs[0], [&](cudaStream_t s) { return new cmg::Solver(descs, s); });
  });
}

int cmg_forest_size(const cmg_hierarchy* h, int* nh) {
  return guard([&]() {
    if (!h || !h->solver || !nh) throw std::invalid_argument("cmg: null argument");
    *nh = h->solver->numHierarchies();
  });
}

int cmg_forest_cells(const cmg_hierarchy* h, int k, int level, int64_t* out) {
  return guard([&]() {
    if (!h || !h->solver || !out) throw std::invalid_argument("cmg: null argument");
    *out = h->solver->hierarchyCells(k, level);
  });
}

int cmg_forest_fill_synthetic(cmg_hierarchy* h, const uint64_t* seeds) {
  return guard([&]() {
    if (!h || !h->solver || !seeds) throw std::invalid_argument("cmg: null argument");
    h->solver->fillSyntheticForest(std::vector<uint64_t>(seeds, seeds + h->solver->numHierarchies()));
  });
}

int cmg_forest_solve(cmg_hierarchy* h, const cmg_solve_params* p, int zero_phi, int mixed, int* exit_status,
                     int* iterations, double* final_norm) {
  return guard([&]() {
    if (!h || !h->solver || !p || !exit_status || !iterations) throw std::invalid_argument("cmg: null argument");
    const std::vector<cmg::SolveResult> r = h->solver->solveForest(solverParams(p), zero_phi != 0, mixed != 0);
    int diverged = -1;
    for (size_t k = 0; k < r.size(); ++k) {
      exit_status[k] = r[k].exitStatus;
      iterations[k] = r[k].iterations;
      if (final_norm) final_norm[k] = r[k].history.back();
      if (r[k].diverged && diverged < 0) diverged = r[k].iterations;
    }
    if (diverged >= 0) throw Diverged(diverged);
  });
}

int cmg_hierarchy_destroy(cmg_hierarchy* h) {
  return guard([&]() {
    if (!h) return;
    delete h->solver;
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
  });
}

int cmg_num_levels(const cmg_hierarchy* h, int* out) {
  return guard([&]() {
    needLevel(h, 0);
    *out = h->solver->numLevels();
  });
}

int cmg_num_boxes(const cmg_hierarchy* h, int level, int* out) {
  return guard([&]() {
    needLevel(h, level);
    *out = (int)h->solver->level(level).grids.size();
  });
}

int cmg_get_boxes(const cmg_hierarchy* h, int level, cmg_box* out, int cap) {
  return guard([&]() {
    needLevel(h, level);
    const auto& g = h->solver->level(level).grids;
    if (!out || cap < (int)g.size()) throw std::invalid_argument("cmg: box buffer too small");
    for (size_t b = 0; b < g.size(); ++b) fromBox(g[b], out[b]);
  });
}

int cmg_num_cells(const cmg_hierarchy* h, int level, int64_t* out) {
  return guard([&]() {
    needLevel(h, level);
    *out = h->solver->numValidCells(level);
  });
}

int cmg_num_faces(const cmg_hierarchy* h, int level, int dir, int64_t* out) {
  return guard([&]() {
    needLevel(h, level);
    if (dir < 0 || dir > 2) throw std::invalid_argument("cmg: direction out of range");
    *out = h->solver->numFaces(level, dir);
  });
}

int cmg_set_rhs(cmg_hierarchy* h, int level, const double* data, int on_device) {
  return guard([&]() {
    needLevel(h, level);
    if (!data) throw std::invalid_argument("cmg: null data");
    h->solver->setRHS(level, data, on_device != 0);
  });
}

int cmg_set_acoef(cmg_hierarchy* h, int level, const double* data, int on_device) {
  return guard([&]() {
    needLevel(h, level);
    if (!data) throw std::invalid_argument("cmg: null data");
    if (!h->desc.vc) throw std::invalid_argument("cmg: operator has no a coefficient");
    h->solver->setACoef(level, data, on_device != 0);
  });
}

int cmg_set_bcoef(cmg_hierarchy* h, int level, int dir, const double* data, int on_device) {
  return guard([&]() {
    needLevel(h, level);
    if (!data || dir < 0 || dir > 2) throw std::invalid_argument("cmg: bad b coefficient argument");
    if (!h->desc.vc) throw std::invalid_argument("cmg: operator has no b coefficient");
    h->solver->setBCoef(level, dir, data, on_device != 0);
  });
}

int cmg_finalize_coefficients(cmg_hierarchy* h) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->finalizeCoefficients();
  });
}

int cmg_get_phi(cmg_hierarchy* h, int level, double* data, int on_device) {
  return guard([&]() {
    needLevel(h, level);
    if (!data) throw std::invalid_argument("cmg: null data");
    h->solver->getPhi(level, data, on_device != 0);
  });
}

int cmg_get_rhs(cmg_hierarchy* h, int level, double* data, int on_device) {
  return guard([&]() {
    needLevel(h, level);
    if (!data) throw std::invalid_argument("cmg: null data");
    h->solver->getRHS(level, data, on_device != 0);
  });
}

int cmg_set_phi(cmg_hierarchy* h, int level, const double* data, int on_device) {
  return guard([&]() {
    needLevel(h, level);
    if (!data) throw std::invalid_argument("cmg: null data");
    h->solver->setPhi(level, data, on_device != 0);
  });
}

namespace {
cmg::SolveParams solverParams(const cmg_solve_params* p) {
  if (!p) throw std::invalid_argument("cmg: null parameters");
  cmg::SolveParams sp;
  sp.pre = p->pre;
  sp.post = p->post;
  sp.bottom = p->bottom;
  sp.numMG = p->num_mg;
  sp.iterMax = p->iter_max;
  sp.imin = p->imin;
  sp.eps = p->eps;
  sp.hang = p->hang;
  sp.normThresh = p->norm_thresh;
  sp.iterMin = p->iter_min;
  if (sp.pre < 0 || sp.post < 0 || sp.bottom < 0 || sp.numMG < 1 || sp.iterMax < 0)
    throw std::invalid_argument("cmg: invalid solver parameters");
  return sp;
}
}  // namespace

namespace {
int solveWith(cmg_hierarchy* h, const cmg_solve_params* p, int zero_phi, int* exit_status, int* iterations,
              double* history, int history_cap, int* history_len, bool mixed) {
  return guard([&]() {
    needLevel(h, 0);
    const cmg::SolveParams sp = solverParams(p);
    cmg::SolveResult r = mixed ? h->solver->solveMixed(sp, zero_phi != 0) : h->solver->solve(sp, zero_phi != 0);
    if (exit_status) *exit_status = r.exitStatus;
    if (iterations) *iterations = r.iterations;
    int n = (int)r.history.size();
    if (history_len) *history_len = n;
    if (history)
      for (int i = 0; i < n && i < history_cap; ++i) history[i] = r.history[i];
    if (r.diverged) throw Diverged(r.iterations);
  });
}
}  // namespace

int cmg_set_relax_mode(cmg_hierarchy* h, int mode) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->setRelaxMode(mode);
  });
}

int cmg_setup_seconds(const cmg_hierarchy* h, double* plans, double* device) {
  return guard([&]() {
    needLevel(h, 0);
    if (plans) *plans = h->solver->planSeconds();
    if (device) *device = h->solver->deviceSeconds();
  });
}

int cmg_host_blocks(int release, size_t* kept) {
  return guard([&]() {
    if (release) cmg::hostBlockRelease();
    if (kept) *kept = cmg::hostBlockKept();
  });
}

int cmg_set_bottom_grid(cmg_hierarchy* h, int mode, int* on_grid) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->setBottomGrid(mode);
    if (on_grid) *on_grid = h->solver->bottomOnGrid() ? 1 : 0;
  });
}

int cmg_set_bottom_solver(cmg_hierarchy* h, const cmg_bottom_params* p) {
  return guard([&]() {
    needLevel(h, 0);
    if (!p) throw std::invalid_argument("cmg: null argument");
    cmg::BottomConfig c;
    c.kind = p->kind;
    c.imax = p->imax;
    c.numRestarts = p->num_restarts;
    c.normType = p->norm_type;
    c.eps = p->eps;
    c.hang = p->hang;
    c.small = p->small;
    h->solver->setBottomConfig(c);
  });
}

int cmg_relax_variants(cmg_hierarchy* h, int* inline_out, float* ms_fill, float* ms_inline, int cap, int* n) {
  return guard([&]() {
    needLevel(h, 0);
    if (!n) throw std::invalid_argument("cmg: null output pointer");
    std::vector<int> v;
    std::vector<float> a, b;
    h->solver->relaxVariants(v, a, b);
    *n = (int)v.size();
    for (int i = 0; i < (int)v.size() && i < cap; ++i) {
      if (inline_out) inline_out[i] = v[i];
      if (ms_fill) ms_fill[i] = i < (int)a.size() ? a[i] : -1.0f;
      if (ms_inline) ms_inline[i] = i < (int)b.size() ? b[i] : -1.0f;
    }
  });
}

int cmg_use_graphs(cmg_hierarchy* h, int on) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->setUseGraphs(on != 0);
  });
}

int cmg_solve(cmg_hierarchy* h, const cmg_solve_params* p, int zero_phi, int* exit_status, int* iterations,
              double* history, int history_cap, int* history_len) {
  return solveWith(h, p, zero_phi, exit_status, iterations, history, history_cap, history_len, false);
}

int cmg_solve_mixed(cmg_hierarchy* h, const cmg_solve_params* p, int zero_phi, int* exit_status, int* iterations,
                    double* history, int history_cap, int* history_len) {
  return solveWith(h, p, zero_phi, exit_status, iterations, history, history_cap, history_len, true);
}

int cmg_set_alpha_beta(cmg_hierarchy* h, double alpha, double beta) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->setAlphaAndBeta(alpha, beta);
  });
}


int cmg_tga(cmg_hierarchy* h, const cmg_solve_params* p, double dt, int nsteps, int* exit_status,
            int* iterations) {
  return guard([&]() {
    needLevel(h, 0);
    if (nsteps < 0 || !(dt > 0)) throw std::invalid_argument("cmg: invalid time step");
    std::vector<cmg::SolveResult> r = h->solver->tga(solverParams(p), dt, nsteps);
    for (size_t n = 0; n < r.size(); ++n) {
      if (exit_status) exit_status[n] = r[n].exitStatus;
      if (iterations) iterations[n] = r[n].iterations;
    }
  });
}

int cmg_backward_euler(cmg_hierarchy* h, const cmg_solve_params* p, double dt, int nsteps, int zero_phi,
                       int* exit_status, int* iterations) {
  return guard([&]() {
    needLevel(h, 0);
    if (nsteps < 0 || !(dt > 0)) throw std::invalid_argument("cmg: invalid time step");
    const cmg::SolveParams sp = solverParams(p);
    std::vector<cmg::SolveResult> r = h->solver->backwardEuler(sp, dt, nsteps, zero_phi != 0);
    for (int n = 0; n < nsteps; ++n) {
      if (exit_status) exit_status[n] = r[n].exitStatus;
      if (iterations) iterations[n] = r[n].iterations;
    }
  });
}

int cmg_solve_multilevel_bicgstab(cmg_hierarchy* h, const cmg_mlsolve_params* p, int zero_phi, int* exit_status,
                                  int* iterations, double* initial_residual, double* final_residual, double* history,
                                  int history_cap, int* history_len) {
  return guard([&]() {
    needLevel(h, 0);
    if (!p) throw std::invalid_argument("cmg: null parameters");
    cmg::MLSolveParams mp;
    mp.mgIters = p->mg_iters;
    mp.mgSmooth = p->mg_smooth;
    mp.imax = p->imax;
    mp.numRestarts = p->num_restarts;
    mp.eps = p->eps;
    mp.reps = p->reps;
    mp.hang = p->hang;
    mp.small = p->small;
    cmg::MLSolveResult r = h->solver->solveMultilevelBiCGStab(mp, zero_phi != 0);
    if (exit_status) *exit_status = r.exitStatus;
    if (iterations) *iterations = r.iterations;
    if (initial_residual) *initial_residual = r.initialResidual;
    if (final_residual) *final_residual = r.finalResidual;
    const int n = (int)r.history.size();
    if (history_len) *history_len = n;
    if (history)
      for (int i = 0; i < n && i < history_cap; ++i) history[i] = r.history[i];
  });
}

int cmg_interp_to_fine(cmg_hierarchy* h, int level, int piecewise_constant) {
  return guard([&]() {
    needLevel(h, level);
    h->solver->interpToFine(level, piecewise_constant != 0);
  });
}

int cmg_fine_interp_destroy(cmg_fine_interp* fi) {
  return guard([&]() {
    if (!fi) return;
    if (fi->work && fi->work != fi->stream) cudaStreamSynchronize(fi->work);
    delete fi->op;
    if (fi->mem) cudaFreeAsync(fi->mem, fi->stream);
    if (fi->stream) {
      cudaStreamSynchronize(fi->stream);
      cudaStreamDestroy(fi->stream);
    }
    delete fi;
  });
}

int cmg_fine_interp_create(const int fine_domain_lo[3], const int fine_domain_hi[3], int nfine, const cmg_box* fine,
                           int ncoarse, const cmg_box* coarse, cmg_fine_interp** out) {
  return guard([&]() {
    if (!fine_domain_lo || !fine_domain_hi || !fine || !coarse || !out || nfine < 1 || ncoarse < 1)
      throw std::invalid_argument("cmg: invalid fine interpolation description");
    *out = nullptr;
    cmg::Box fdom(cmg::IV(fine_domain_lo[0], fine_domain_lo[1], fine_domain_lo[2]),
                  cmg::IV(fine_domain_hi[0], fine_domain_hi[1], fine_domain_hi[2]));
    if (fdom.empty() || !fdom.coarsenable(2)) throw std::invalid_argument("cmg: fine domain empty or not coarsenable by 2");
    const cmg::Box cdom = fdom.coarsen(2);
    std::vector<cmg::Box> fb, cb;
    for (int b = 0; b < nfine; ++b) {
      cmg::Box x = toBox(fine[b]);
      if (x.empty() || !fdom.contains(x) || !x.coarsenable(2))
        throw std::invalid_argument("cmg: fine box empty, outside the fine domain or not coarsenable by 2");
      fb.push_back(x);
    }
    for (int b = 0; b < ncoarse; ++b) {
      cmg::Box x = toBox(coarse[b]);
      if (x.empty() || !cdom.contains(x)) throw std::invalid_argument("cmg: coarse box empty or outside the domain");
      cb.push_back(x);
    }
    cmg::BoxIndex cindex;
    cindex.build(cb);
    std::vector<cmg::FlatBox> cf, ff;
    cmg_fine_interp* fi = new cmg_fine_interp;
    fi->ncoarse = cmg::flatBoxes(cb, cf);
    fi->nfine = cmg::flatBoxes(fb, ff);
    try {
      cudaError_t e = cudaStreamCreateWithFlags(&fi->stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) throw std::runtime_error(std::string("cmg: stream: ") + cudaGetErrorString(e));
      fi->work = fi->stream;
      fi->op = new cmg::FineInterpOp(cb, cindex, cdom, fb, fi->stream);
      auto up = [](size_t n) { return (n + 255) & ~(size_t)255; };
      const size_t cB = up(cf.size() * sizeof(cmg::FlatBox)), fB = up(ff.size() * sizeof(cmg::FlatBox));
      const size_t dC = up(fi->ncoarse * sizeof(double)), dF = up(fi->nfine * sizeof(double));
      e = cudaMallocAsync(&fi->mem, cB + fB + dC + dF, fi->stream);
      if (e != cudaSuccess) throw std::runtime_error(std::string("cmg: cudaMalloc fine interpolation: ") + cudaGetErrorString(e));
      char* p = (char*)fi->mem;
      std::vector<char> host(cB + fB);
      std::memcpy(host.data(), cf.data(), cf.size() * sizeof(cmg::FlatBox));
      std::memcpy(host.data() + cB, ff.data(), ff.size() * sizeof(cmg::FlatBox));
      e = cudaMemcpyAsync(p, host.data(), host.size(), cudaMemcpyHostToDevice, fi->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(fi->stream);
      if (e != cudaSuccess) throw std::runtime_error(std::string("cmg: fine interpolation tables: ") + cudaGetErrorString(e));
      fi->cflat = (const cmg::FlatBox*)p;
      fi->fflat = (const cmg::FlatBox*)(p + cB);
      fi->dcoarse = (double*)(p + cB + fB);
      fi->dfine = (double*)(p + cB + fB + dC);
    } catch (...) {
      cmg_fine_interp_destroy(fi);
      throw;
    }
    *out = fi;
  });
}

int cmg_fine_interp_run(cmg_fine_interp* fi, const double* coarse, double* fine, int on_device,
                        int piecewise_constant) {
  return guard([&]() {
    if (!fi || !fi->op || !coarse || !fine) throw std::invalid_argument("cmg: null fine interpolation argument");
    const bool pwc = piecewise_constant != 0;
    auto ck = [](cudaError_t e, const char* what) {
      if (e != cudaSuccess) throw std::runtime_error(std::string("cmg: ") + what + ": " + cudaGetErrorString(e));
    };
    const double* c = coarse;
    double* f = fine;
    if (!on_device) {
      ck(cudaMemcpyAsync(fi->dcoarse, coarse, fi->ncoarse * sizeof(double), cudaMemcpyHostToDevice, fi->work),
         "fine interpolation h2d");
      c = fi->dcoarse;
      f = fi->dfine;
    }
    fi->op->runFlat(fi->cflat, c, fi->fflat, f, pwc);
    if (!on_device)
      ck(cudaMemcpyAsync(fine, fi->dfine, fi->nfine * sizeof(double), cudaMemcpyDeviceToHost, fi->work),
         "fine interpolation d2h");
    ck(cudaStreamSynchronize(fi->work), "fine interpolation sync");
  });
}

int cmg_residual_norm(cmg_hierarchy* h, double* out) {
  return guard([&]() {
    needLevel(h, 0);
    *out = h->solver->residualNorm();
  });
}

static_assert(CMG_NOALLOC_MAX_BOXES == cmg::NOALLOC_MAX_BOXES, "header limit matches the scratch size");

int cmg_residual_norm_noalloc(cmg_hierarchy* h, double* out) {
  return guard([&]() {
    needLevel(h, 0);
    if (!out) throw std::invalid_argument("cmg: null output pointer");
    *out = cmg::residualNormNoAlloc(*h->solver);
  });
}

int cmg_residual_norm_noalloc_forget(void) {
  return guard([&]() { cmg::forgetNoAllocScratch(); });
}

static int syntheticHierarchyImpl(int n0, int nlevels, int max_box, int block_factor, double fill_ratio,
                                  uint64_t seed, double thresh, int* nlevels_out, int* nboxes, cmg_box* boxes,
                                  int cap, int* ntotal, bool device) {
  return guard([&]() {
    if (!nlevels_out || !nboxes || !ntotal) throw std::invalid_argument("cmg: null output pointer");
    if (max_box < 0 || block_factor < 1 || !(fill_ratio > 0.0 && fill_ratio <= 1.0))
      throw std::invalid_argument("cmg: invalid grid generation parameters");
    std::vector<std::vector<cmg::Box>> g;
    if (device) {
      cudaStream_t s = nullptr;
      if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        throw std::runtime_error("cmg: no CUDA device for tagging");
      try {
        cmg::DeviceTagger tagger(s);
        g = cmg::syntheticHierarchy(n0, nlevels, max_box, block_factor, fill_ratio, seed, thresh, &tagger);
      } catch (...) {
        cudaStreamDestroy(s);
        throw;
      }
      cudaStreamDestroy(s);
    } else {
      g = cmg::syntheticHierarchy(n0, nlevels, max_box, block_factor, fill_ratio, seed, thresh);
    }
    *nlevels_out = (int)g.size();
    int total = 0;
    for (size_t l = 0; l < g.size(); ++l) {
      nboxes[l] = (int)g[l].size();
      for (const cmg::Box& b : g[l]) {
        if (boxes && total < cap) fromBox(b, boxes[total]);
        ++total;
      }
    }
    *ntotal = total;
  });
}

int cmg_synthetic_hierarchy(int n0, int nlevels, int max_box, int block_factor, double fill_ratio, uint64_t seed,
                            double thresh, int* nlevels_out, int* nboxes, cmg_box* boxes, int cap, int* ntotal) {
  return syntheticHierarchyImpl(n0, nlevels, max_box, block_factor, fill_ratio, seed, thresh, nlevels_out, nboxes,
                                boxes, cap, ntotal, false);
}

int cmg_synthetic_hierarchy_device(int n0, int nlevels, int max_box, int block_factor, double fill_ratio,
                                   uint64_t seed, double thresh, int* nlevels_out, int* nboxes, cmg_box* boxes,
                                   int cap, int* ntotal) {
  return syntheticHierarchyImpl(n0, nlevels, max_box, block_factor, fill_ratio, seed, thresh, nlevels_out, nboxes,
                                boxes, cap, ntotal, true);
}

int cmg_serve(const cmg_request* reqs, int n, double hbm_budget, int max_inflight, int open_loop,
              cmg_request_result* out, double* wall_seconds) {
  return cmg_serve_batched(reqs, n, hbm_budget, max_inflight, open_loop, 0.0, 1, out, wall_seconds);
}

int cmg_serve_batched(const cmg_request* reqs, int n, double hbm_budget, int max_inflight, int open_loop,
                      double batch_window, int max_batch, cmg_request_result* out, double* wall_seconds) {
  return guard([&]() {
    if ((!reqs && n > 0) || (!out && n > 0) || n < 0 || max_inflight < 1 || !(hbm_budget > 0) ||
        !(batch_window >= 0) || max_batch < 1)
      throw std::invalid_argument("cmg: invalid serve arguments");
    std::vector<cmg::Request> rq(n);
    for (int i = 0; i < n; ++i) {
      const cmg_request& a = reqs[i];
      cmg::Request& r = rq[i];
      r.arrival = a.arrival;
      r.n0 = a.n0;
      r.levels = a.levels;
      r.maxBox = a.max_box;
      r.blockFactor = a.block_factor;
      r.fillRatio = a.fill_ratio;
      r.thresh = a.thresh;
      r.seed = a.seed;
      r.op = a.op;
      r.alpha = a.alpha;
      r.beta = a.beta;
      r.params.pre = a.params.pre;
      r.params.post = a.params.post;
      r.params.bottom = a.params.bottom;
      r.params.numMG = a.params.num_mg;
      r.params.iterMax = a.params.iter_max;
      r.params.imin = a.params.imin;
      r.params.eps = a.params.eps;
      r.params.hang = a.params.hang;
      r.params.normThresh = a.params.norm_thresh;
      r.params.iterMin = a.params.iter_min;
      r.mixed = a.mixed != 0;
      r.graphs = a.graphs != 0;
      r.deviceTags = a.device_tags != 0;
      r.timeout = a.timeout;
      r.cancel = a.cancel;
      r.injectNanRHS = a.inject_nan_rhs != 0;
      r.injectCancelAfter = a.inject_cancel_after;
    }
    cmg::ServeOptions opt;
    opt.hbmBudget = hbm_budget;
    opt.maxInflight = max_inflight;
    opt.openLoop = open_loop != 0;
    opt.batchWindow = batch_window;
    opt.maxBatch = max_batch;
    std::vector<cmg::RequestResult> res;
    double wall = cmg::serve(rq, opt, res);
    if (wall_seconds) *wall_seconds = wall;
    for (int i = 0; i < n; ++i) {
      const cmg::RequestResult& a = res[i];
      cmg_request_result& o = out[i];
      o.exit_status = a.exitStatus;
      o.iterations = a.iterations;
      o.error = a.error;
      o.admitted = a.admitted;
      o.started = a.started;
      o.solved = a.solved;
      o.finished = a.finished;
      o.setup_seconds = a.setupSeconds;
      o.solve_seconds = a.solveSeconds;
      o.r0 = a.r0;
      o.rfinal = a.rfinal;
      o.grid_seconds = a.gridSeconds;
      o.build_seconds = a.buildSeconds;
      o.batch_size = a.batchSize;
      o.fill_seconds = a.fillSeconds;
      o.cells = a.cells;
      o.estimate_bytes = a.estimate;
      std::snprintf(o.message, sizeof(o.message), "%s", a.message.c_str());
      o.device_bytes = a.deviceBytes;
      o.phi_hash = a.phiHash;
    }
  });
}

int cmg_fill_synthetic_device(cmg_hierarchy* h, uint64_t seed) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->fillSyntheticDevice(seed);
  });
}

int cmg_fill_synthetic(cmg_hierarchy* h, uint64_t seed) {
  return guard([&]() {
    needLevel(h, 0);
    cmg::fillSynthetic(*h->solver, h->desc.vc != 0, seed);
  });
}

int cmg_domain_split(const int domain_lo[3], const int domain_hi[3], int max_box, int block_factor, cmg_box* out,
                     int cap, int* n) {
  return guard([&]() {
    if (!domain_lo || !domain_hi || !n || block_factor < 1 || max_box < 0)
      throw std::invalid_argument("cmg: invalid domainSplit arguments");
    cmg::Box dom(cmg::IV(domain_lo[0], domain_lo[1], domain_lo[2]), cmg::IV(domain_hi[0], domain_hi[1], domain_hi[2]));
    if (!dom.coarsenable(block_factor)) throw std::invalid_argument("cmg: domain not coarsenable by the blocking factor");
    cmg::Layout l(cmg::domainSplit(dom, max_box, block_factor));
    *n = (int)l.size();
    if (out) {
      if (cap < (int)l.size()) throw std::invalid_argument("cmg: box buffer too small");
      for (size_t b = 0; b < l.size(); ++b) fromBox(l[b], out[b]);
    }
  });
}

int cmg_exchange_plan(const cmg_hierarchy* h, int level, int* items14, int cap, int* n) {
  return guard([&]() {
    needLevel(h, level);
    auto plan = cmg::exchangePlan(h->solver->level(level).grids);
    *n = (int)plan.size();
    if (items14) {
      if (cap < (int)plan.size()) throw std::invalid_argument("cmg: item buffer too small");
      for (size_t i = 0; i < plan.size(); ++i)
        putMotion(items14 + 14 * i, plan[i].from, plan[i].to, plan[i].fromRegion, plan[i].toRegion);
    }
  });
}

int cmg_coarse_fine_plan(const cmg_hierarchy* h, int level, int* items14, int cap, int* n) {
  return guard([&]() {
    needLevel(h, level);
    if (level < 1) throw std::invalid_argument("cmg: level 0 has no coarser level");
    const auto& F = h->solver->level(level);
    *n = (int)F.toCoarse.size();
    if (items14) {
      if (cap < *n) throw std::invalid_argument("cmg: item buffer too small");
      for (size_t i = 0; i < F.toCoarse.size(); ++i) {
        const auto& it = F.toCoarse[i];
        cmg::Box r(cmg::IV(it.lo[0], it.lo[1], it.lo[2]), cmg::IV(it.hi[0], it.hi[1], it.hi[2]));
        putMotion(items14 + 14 * i, it.fbox, it.cbox, r, r);
      }
    }
  });
}

int cmg_get_stream(const cmg_hierarchy* h, void** stream) {
  return guard([&]() {
    needLevel(h, 0);
    if (!stream) throw std::invalid_argument("cmg: null output");
    *stream = (void*)h->solver->stream();
  });
}

int cmg_set_stream(cmg_hierarchy* h, void* stream) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->setStream((cudaStream_t)stream);
  });
}

int cmg_fine_interp_set_stream(cmg_fine_interp* fi, void* stream) {
  return guard([&]() {
    if (!fi || !fi->op) throw std::invalid_argument("cmg: null fine interpolation");
    cudaStream_t s = stream ? (cudaStream_t)stream : fi->stream;
    if (s == fi->work) return;
    cudaError_t e = cudaStreamSynchronize(fi->work);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cmg: stream switch: ") + cudaGetErrorString(e));
    fi->work = s;
    fi->op->setStream(s);
  });
}

int cmg_fine_interp_is_fused(const cmg_fine_interp* fi, int* out) {
  return guard([&]() {
    if (!fi || !fi->op || !out) throw std::invalid_argument("cmg: null fine interpolation argument");
    *out = fi->op->fused() ? 1 : 0;
  });
}

// ---------------------------------------------------------------- operator-level calls

namespace {
cmg::Solver& opSolver(cmg_hierarchy* h, int lev) {
  needLevel(h, 0);
  h->solver->opPlan(lev);  // range check
  return *h->solver;
}
const cmg::Solver& opSolverC(const cmg_hierarchy* h, int lev) {
  needLevel(h, 0);
  h->solver->opPlan(lev);
  return *h->solver;
}
void needPtr(const void* p) {
  if (!p) throw std::invalid_argument("cmg: null operator argument");
}
}  // namespace

int cmg_op_num_mg_depths(const cmg_hierarchy* h, int* out) {
  return guard([&]() {
    needLevel(h, 0);
    needPtr(out);
    *out = h->solver->numMGDepths();
  });
}

int cmg_op_num_boxes(const cmg_hierarchy* h, int lev, int* out) {
  return guard([&]() {
    needPtr(out);
    *out = (int)opSolverC(h, lev).opPlan(lev).grids.size();
  });
}

int cmg_op_get_boxes(const cmg_hierarchy* h, int lev, cmg_box* out, int cap) {
  return guard([&]() {
    needPtr(out);
    const cmg::Layout& g = opSolverC(h, lev).opPlan(lev).grids;
    if (cap < (int)g.size()) throw std::invalid_argument("cmg: box buffer too small");
    for (size_t b = 0; b < g.size(); ++b) fromBox(g[b], out[b]);
  });
}

int cmg_op_size(const cmg_hierarchy* h, int lev, int64_t* out) {
  return guard([&]() {
    needPtr(out);
    *out = opSolverC(h, lev).opSize(lev);
  });
}

int cmg_op_coarsened_size(const cmg_hierarchy* h, int level, int64_t* out) {
  return guard([&]() {
    needPtr(out);
    *out = opSolverC(h, level).opCoarsenedSize(level);
  });
}

int cmg_op_residual(cmg_hierarchy* h, int lev, double* lhs, const double* phi, const double* rhs, int homogeneous) {
  return guard([&]() {
    needPtr(lhs);
    opSolver(h, lev).opResidual(lev, lhs, phi, rhs, homogeneous != 0);
  });
}

int cmg_op_apply(cmg_hierarchy* h, int lev, double* lhs, const double* phi, int homogeneous) {
  return guard([&]() {
    needPtr(lhs);
    opSolver(h, lev).opApply(lev, lhs, phi, homogeneous != 0);
  });
}

int cmg_op_relax(cmg_hierarchy* h, int lev, double* phi, const double* rhs, int iterations) {
  return guard([&]() {
    if (iterations < 0) throw std::invalid_argument("cmg: negative relaxation count");
    opSolver(h, lev).opRelax(lev, phi, rhs, iterations);
  });
}

int cmg_op_precond(cmg_hierarchy* h, int lev, double* cor, const double* res) {
  return guard([&]() { opSolver(h, lev).opPreCond(lev, cor, res); });
}

int cmg_op_restrict_residual(cmg_hierarchy* h, int lev, double* res_coarse, const double* phi, const double* rhs) {
  return guard([&]() { opSolver(h, lev).opRestrictResidual(lev, res_coarse, phi, rhs); });
}

int cmg_op_prolong_increment(cmg_hierarchy* h, int lev, double* phi, const double* corr_coarse) {
  return guard([&]() { opSolver(h, lev).opProlongIncrement(lev, phi, corr_coarse); });
}

int cmg_op_amr_operator(cmg_hierarchy* h, int level, int form, double* out, const double* phi_fine,
                        double* phi, const double* phi_coarse, const double* rhs) {
  return guard([&]() {
    needPtr(out);
    opSolver(h, level).opAMROperator(level, out, phi_fine, phi, phi_coarse, rhs, form);
  });
}

int cmg_op_amr_restrict(cmg_hierarchy* h, int level, double* res_coarsened, const double* residual,
                        const double* correction, const double* coarse_correction) {
  return guard([&]() {
    needPtr(res_coarsened);
    if (correction) needPtr(coarse_correction);
    opSolver(h, level).opAMRRestrict(level, res_coarsened, residual, correction, coarse_correction);
  });
}

int cmg_op_assign_coarsened(cmg_hierarchy* h, int level, double* coarse, const double* coarsened) {
  return guard([&]() {
    needPtr(coarsened);
    opSolver(h, level).opAssignCoarsened(level, coarse, coarsened);
  });
}

int cmg_op_amr_prolong(cmg_hierarchy* h, int level, double* correction, const double* coarse_correction) {
  return guard([&]() { opSolver(h, level).opAMRProlong(level, correction, coarse_correction); });
}

int cmg_op_amr_update_residual(cmg_hierarchy* h, int level, double* residual, const double* correction,
                               const double* coarse_correction) {
  return guard([&]() { opSolver(h, level).opAMRUpdateResidual(level, residual, correction, coarse_correction); });
}

int cmg_op_cf_interp(cmg_hierarchy* h, int level, double* phi, const double* phi_coarse) {
  return guard([&]() {
    needPtr(phi_coarse);
    opSolver(h, level).opCFInterp(level, phi, phi_coarse);
  });
}

int cmg_op_zero_covered(cmg_hierarchy* h, int level, double* data) {
  return guard([&]() { opSolver(h, level).opZeroCovered(level, data); });
}

int cmg_op_axby(cmg_hierarchy* h, int lev, double* lhs, const double* x, const double* y, double a, double b) {
  return guard([&]() {
    needPtr(lhs);
    needPtr(x);
    needPtr(y);
    opSolver(h, lev).opAxby(lev, lhs, x, y, a, b);
  });
}

int cmg_op_incr(cmg_hierarchy* h, int lev, double* lhs, const double* x, double scale) {
  return guard([&]() {
    needPtr(lhs);
    needPtr(x);
    opSolver(h, lev).opIncr(lev, lhs, x, scale);
  });
}

int cmg_op_scale(cmg_hierarchy* h, int lev, double* lhs, double scale) {
  return guard([&]() {
    needPtr(lhs);
    opSolver(h, lev).opScale(lev, lhs, scale);
  });
}

int cmg_op_dot(cmg_hierarchy* h, int lev, const double* x, const double* y, double* out) {
  return guard([&]() {
    needPtr(out);
    *out = opSolver(h, lev).opDot(lev, x, y);
  });
}

int cmg_op_norm(cmg_hierarchy* h, int lev, const double* x, int ord, double* out) {
  return guard([&]() {
    needPtr(out);
    *out = opSolver(h, lev).opNorm(lev, x, ord);
  });
}

int cmg_launch_count(int64_t* out) {
  return guard([&]() {
    if (!out) throw std::invalid_argument("cmg: null output");
    *out = (int64_t)cmg::launchCount();
  });
}

int cmg_profile_enable(cmg_hierarchy* h, int on) {
  return guard([&]() {
    needLevel(h, 0);
    h->solver->profileEnable(on != 0);
  });
}

int cmg_profile_read(cmg_hierarchy* h, int kernel_class, int64_t* launches, double* ms, double* bytes) {
  return guard([&]() {
    needLevel(h, 0);
    if (!launches || !ms || !bytes) throw std::invalid_argument("cmg: null output");
    h->solver->profileRead(kernel_class, launches, ms, bytes);
  });
}

int cmg_layout_exchange_plan(const cmg_box* boxes, int nbox, int* items14, int cap, int* n) {
  return guard([&]() {
    if (!boxes || nbox < 1 || !n) throw std::invalid_argument("cmg: invalid box list");
    std::vector<cmg::Box> v;
    for (int b = 0; b < nbox; ++b) v.push_back(toBox(boxes[b]));
    auto plan = cmg::exchangePlan(cmg::Layout(v));
    *n = (int)plan.size();
    if (items14) {
      if (cap < (int)plan.size()) throw std::invalid_argument("cmg: item buffer too small");
      for (size_t i = 0; i < plan.size(); ++i)
        putMotion(items14 + 14 * i, plan[i].from, plan[i].to, plan[i].fromRegion, plan[i].toRegion);
    }
  });
}

int cmg_layout_exchange_plan_periodic(const cmg_box* boxes, int nbox, const cmg_box* domain, const int* periodic,
                                      int* items14, int cap, int* n) {
  return guard([&]() {
    if (!boxes || nbox < 1 || !domain || !periodic || !n) throw std::invalid_argument("cmg: invalid box list");
    std::vector<cmg::Box> v;
    for (int b = 0; b < nbox; ++b) v.push_back(toBox(boxes[b]));
    const bool per[3] = {periodic[0] != 0, periodic[1] != 0, periodic[2] != 0};
    auto plan = cmg::exchangePlan(cmg::Layout(v), toBox(*domain), per);
    *n = (int)plan.size();
    if (items14) {
      if (cap < (int)plan.size()) throw std::invalid_argument("cmg: item buffer too small");
      for (size_t i = 0; i < plan.size(); ++i)
        putMotion(items14 + 14 * i, plan[i].from, plan[i].to, plan[i].fromRegion, plan[i].toRegion);
    }
  });
}

int cmg_layout_coarse_fine_plan(const cmg_box* fine, int nfine, const cmg_box* coarse, int ncoarse, int* items14,
                                int cap, int* n) {
  return guard([&]() {
    if (!fine || !coarse || nfine < 1 || ncoarse < 1 || !n) throw std::invalid_argument("cmg: invalid box lists");
    std::vector<cmg::Box> f, c;
    for (int b = 0; b < nfine; ++b) f.push_back(toBox(fine[b]));
    for (int b = 0; b < ncoarse; ++b) c.push_back(toBox(coarse[b]));
    auto plan = cmg::copyPlan(cmg::Layout(f).coarsen(2), cmg::Layout(c));
    *n = (int)plan.size();
    if (items14) {
      if (cap < (int)plan.size()) throw std::invalid_argument("cmg: item buffer too small");
      for (size_t i = 0; i < plan.size(); ++i)
        putMotion(items14 + 14 * i, plan[i].from, plan[i].to, plan[i].fromRegion, plan[i].toRegion);
    }
  });
}

int cmg_vcycle_bytes(const cmg_hierarchy* h, const cmg_solve_params* p, double* out) {
  return guard([&]() {
    needLevel(h, 0);
    cmg::SolveParams sp;
    sp.pre = p->pre;
    sp.post = p->post;
    *out = h->solver->vcycleBytes(sp);
  });
}

}  // extern "C"
