/*
 * cmg.h -- C ABI of the B200 AMR multigrid solve (libcmg.so).
 *
 * This is the boundary a host program binds to replace the reference's
 * AMRMultiGrid<LevelData<FArrayBox>>::solve over AMRPoissonOp /
 * VCAMRPoissonOp2 (Chombo lib/src/AMRElliptic).  Plain pointers and sizes
 * only; every call returns an int status (CMG_OK on success) and never aborts.
 * Field data cross the boundary as the valid cells of every box of a level,
 * boxes in DisjointBoxLayout order (sorted, BoxTools/BoxLayout.cpp:89-119),
 * cells x-fastest inside a box (BaseFab order, BoxTools/BaseFabImplem.H:291-312).
 * Face coefficients in direction d use the face box of each cell box
 * (surroundingNodes, hi[d] + 1).
 */
#ifndef CMG_H
#define CMG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CMG_OK = 0,
  CMG_EINVAL = 1,    /* bad argument (level, direction, sizes, null pointer) */
  CMG_ENOMEM = 2,    /* device allocation failed */
  CMG_ECUDA = 3,     /* CUDA runtime error */
  CMG_EINTERNAL = 4, /* anything else; see cmg_last_error() */
  CMG_EDIVERGED = 5, /* a residual norm became NaN or infinite: the solve stopped there; its outputs
                        (phi, exit status, history up to that norm) are written */
  CMG_ETIMEOUT = 6,  /* a request's time limit passed before it finished (cmg_serve) */
  CMG_ECANCELLED = 7 /* a request was cancelled (cmg_serve) */
};

typedef struct cmg_box {
  int lo[3];
  int hi[3];
} cmg_box;

typedef struct cmg_hierarchy cmg_hierarchy;

/* Solver parameters: AMRMultiGrid::setSolverParameters
 * (AMRElliptic/AMRMultiGrid.H:527-553) plus m_imin and m_iterMin
 * (AMRMultiGrid.H:599-622, 1003-1008).  The reference's defaults are
 * {2, 2, 2, 1, 20, 5, 1e-6, 1e-15, 1e-30, -1}. */
typedef struct cmg_solve_params {
  int pre, post, bottom, num_mg, iter_max, imin;
  double eps, hang, norm_thresh;
  int iter_min; /* iterate while iteration < iter_min whatever the norms (-1: no minimum) */
} cmg_solve_params;

/* Message of the last failed call on this thread. */
const char* cmg_last_error(void);

/* Builds a hierarchy: level-0 domain box, level-0 cell size, per-level box
 * counts and the concatenated boxes (refinement ratio 2 between levels), and
 * the operator.  op = 0: AMRPoissonOp, L = alpha phi + beta Lap(phi)
 * (AMRPoissonOpFactory::define, AMRElliptic/AMRPoissonOp.cpp:1857-1903);
 * op = 1: VCAMRPoissonOp2, L = alpha a phi - beta div(b grad phi)
 * (VCAMRPoissonOp2Factory::define, AMRElliptic/VCAMRPoissonOp2.cpp:873-924).
 * Boundary conditions are homogeneous Dirichlet on every domain face
 * (the examples' ParseBC, releasedExamples/AMRPoisson/execCell/poissonSolve.cpp:76-119);
 * cmg_hierarchy_create_bc takes one per face.
 * Builds every plan (exchange copiers, coarse-fine stencils, flux registers,
 * multigrid levels: AMRMultiGrid::define, AMRMultiGrid.H:1292-1328) and
 * allocates all device state. */
int cmg_hierarchy_create(const int domain_lo[3], const int domain_hi[3], double dx0, int nlevels,
                         const int* nboxes, const cmg_box* boxes, int op, double alpha, double beta,
                         cmg_hierarchy** out);
/* The same with a homogeneous boundary type per domain face, in the order
 * x-lo, x-hi, y-lo, y-hi, z-lo, z-hi: CMG_BC_DIRICHLET (ghost = 2*0 - inside,
 * DiriBC order 1 with value 0, BCFunc.cpp:294-354) or CMG_BC_NEUMANN (ghost =
 * inside, NeumBC with value 0, BCFunc.cpp:217-236), as the AMRINS projection's
 * pressure BC function sets them (walls and inflow Neumann, outflow
 * Dirichlet).  bc == NULL is Dirichlet everywhere.  With Neumann on every
 * face the operator is singular; the solver runs as the reference's does. */
#define CMG_BC_DIRICHLET 0
#define CMG_BC_NEUMANN 1
/* A periodic direction (both of its faces; ProblemDomain's periodicity):
 * ghost cells beyond the domain come from the domain's periodic image.
 * One-level hierarchies only (CMG_EINVAL otherwise). */
#define CMG_BC_PERIODIC 2
int cmg_hierarchy_create_bc(const int domain_lo[3], const int domain_hi[3], double dx0, int nlevels,
                            const int* nboxes, const cmg_box* boxes, int op, double alpha, double beta,
                            const int bc[6], cmg_hierarchy** out);
int cmg_hierarchy_destroy(cmg_hierarchy* h);

/* A forest: nh hierarchies with the same level-0 domain, dx0, level count,
 * operator and boundary types, whose level-0 layouts coarsen alike (the same
 * multigrid depths), solved together: every operation of a V-cycle is one
 * launch over the boxes of all of them (their levels concatenated, each
 * hierarchy in its own element range), the bottom solves one thread block per
 * hierarchy.  nboxes holds nh * nlevels counts (hierarchy by hierarchy, level
 * by level) and boxes the boxes in that order.  The handle is a hierarchy
 * whose level data (cmg_set_rhs, cmg_get_phi, ...) is the hierarchies' data
 * one after the other (cmg_forest_cells gives each part); solve it with
 * cmg_forest_solve.  The single-hierarchy solves, operators and FineInterp
 * refuse a forest with CMG_EINVAL. */
int cmg_forest_create(int nh, const int domain_lo[3], const int domain_hi[3], double dx0, int nlevels,
                      const int* nboxes, const cmg_box* boxes, int op, double alpha, double beta, const int bc[6],
                      cmg_hierarchy** out);
int cmg_forest_size(const cmg_hierarchy* h, int* nh);
/* Valid cells of hierarchy k on a level. */
int cmg_forest_cells(const cmg_hierarchy* h, int k, int level, int64_t* out);
/* cmg_fill_synthetic (device generator) of every hierarchy, seeds[k] for hierarchy k. */
int cmg_forest_fill_synthetic(cmg_hierarchy* h, const uint64_t* seeds);
/* AMRMultiGrid::solve of every hierarchy of the forest at once (mixed != 0:
 * FP32 V-cycles in FP64 refinement, as cmg_solve_mixed): each hierarchy keeps
 * its own residual norm, stopping rule and bottom-solver metric, and its phi
 * takes no correction after its own stop, so exit_status[k], iterations[k]
 * and phi of hierarchy k are those of its own solve.  final_norm (may be
 * NULL): each hierarchy's last composite residual norm.  CMG_EDIVERGED when a
 * hierarchy's norm became non-finite (the others' results are written). */
int cmg_forest_solve(cmg_hierarchy* h, const cmg_solve_params* p, int zero_phi, int mixed, int* exit_status,
                     int* iterations, double* final_norm);

/* Sizes of the per-level data arrays. */
int cmg_num_levels(const cmg_hierarchy* h, int* out);
int cmg_num_boxes(const cmg_hierarchy* h, int level, int* out);
int cmg_get_boxes(const cmg_hierarchy* h, int level, cmg_box* out, int cap);
int cmg_num_cells(const cmg_hierarchy* h, int level, int64_t* out);
int cmg_num_faces(const cmg_hierarchy* h, int level, int dir, int64_t* out);

/* Right-hand side, coefficients and solution.  on_device != 0: the pointer is
 * device memory of the current device.  Replaces filling the LevelData
 * arguments of AMRMultiGrid::solve (AMRMultiGrid.H:894-904) and the
 * coefficient LevelData of VCAMRPoissonOp2Factory::define. */
int cmg_set_rhs(cmg_hierarchy* h, int level, const double* data, int on_device);
int cmg_set_acoef(cmg_hierarchy* h, int level, const double* data, int on_device);
int cmg_set_bcoef(cmg_hierarchy* h, int level, int dir, const double* data, int on_device);
/* Computes the relaxation coefficient (VCAMRPoissonOp2::resetLambda,
 * VCAMRPoissonOp2.cpp:283-318) and the multigrid coefficient averages
 * (VCAMRPoissonOp2Factory::MGnewOp, VCAMRPoissonOp2.cpp:1019-1058).  Call
 * after the coefficients are set and before cmg_solve (op = 1 only). */
int cmg_finalize_coefficients(cmg_hierarchy* h);
int cmg_get_phi(cmg_hierarchy* h, int level, double* data, int on_device);
int cmg_get_rhs(cmg_hierarchy* h, int level, double* data, int on_device);
int cmg_set_phi(cmg_hierarchy* h, int level, const double* data, int on_device);

/* AMRMultiGrid::solve(phi, rhs, lmax, 0, zeroPhi) (AMRMultiGrid.H:894-1124).
 * history receives the composite max-norm residual at the start of every
 * iteration followed by the final one (up to history_cap values).  A norm
 * that is NaN or infinite (a NaN in the right-hand side, or a diverging
 * iteration) ends the solve there and the call returns CMG_EDIVERGED with
 * every output written; exit_status is the reference's bitmask for that
 * norm (AMRMultiGrid.H:1099). */
int cmg_solve(cmg_hierarchy* h, const cmg_solve_params* p, int zero_phi, int* exit_status, int* iterations,
              double* history, int history_cap, int* history_len);

/* Replays every solver iteration (V-cycle, phi update, composite residual)
 * from a CUDA graph captured on its first use for the given precision and
 * smoothing parameters (no counterpart in the reference).  Same kernels in
 * the same order, so the same results; saves the per-launch host cost.
 * Off by default; profiling (cmg_profile_enable) runs uncaptured. */
int cmg_use_graphs(cmg_hierarchy* h, int on);

/* Relaxation variant (no counterpart in the reference): 0 = chosen per level
 * by a timing autotuner before the first solve (default); 1 = ghost fill
 * (exchange, boundary and coarse-fine values) before each colour pass, as the
 * reference's levelGSRB; 2 = no separate fill: every block of a colour pass
 * first writes the face ghosts its own cells read (the same fill entries),
 * then updates its cells; 3 = fused sweeps: both colours
 * of a sweep in one launch (every box marching through its z slabs, the
 * colour-1 cells on faces shared with another box in a second launch), no
 * fill.  Identical results. */
int cmg_set_relax_mode(cmg_hierarchy* h, int mode);

/* The bottom solver of the deepest multigrid level, as the LinearSolver
 * AMRMultiGrid::define is given: CMG_BOTTOM_BICGSTAB (BiCGStabSolver,
 * BiCGStabSolver.H:199-515; the default, with its defaults imax 80,
 * num_restarts 5, norm_type 2, hang 1e-8, small 1e-30; its tolerance is the
 * one the multigrid solve hands it, so eps is not read) or CMG_BOTTOM_RELAX
 * (RelaxSolver, RelaxSolver.H:128-186: imax corrections by the operator's
 * preconditioner, stopping below eps times the initial residual norm or on a
 * hang; its defaults imax 40, norm_type 2, eps 1e-6, hang 0, the bottom of the
 * AMRINS projection solves).  norm_type 2 or 0. */
#define CMG_BOTTOM_BICGSTAB 0
#define CMG_BOTTOM_RELAX 1
typedef struct cmg_bottom_params {
  int kind, imax, num_restarts, norm_type;
  double eps, hang, small;
} cmg_bottom_params;
int cmg_set_bottom_solver(cmg_hierarchy* h, const cmg_bottom_params* p);
/* Where the bottom solve runs: -1 automatic (the default: across the whole
 * device in one cooperative launch for a single hierarchy whose bottom level
 * has at least 4096 cells, else one thread block per hierarchy), 0 one thread
 * block per hierarchy, 1 the whole device (single hierarchies only; a forest
 * keeps one block per hierarchy).  Identical results.  *on_grid (may be
 * null) receives 1 when the grid-wide solve is in use. */
int cmg_set_bottom_grid(cmg_hierarchy* h, int mode, int* on_grid);
/* The relaxation variant of every AMR level, then every multigrid depth
 * (0 = ghost fills, 1 = in-pass ghosts, 2 = all sweeps in one one-block
 * launch, for levels of at most 32768 cells, 3 = fused sweeps), with the autotuner's times in
 * ms for four sweeps with fills and with the best other variant (-1 when a
 * mode was forced); runs the tuner if it has not run.  n: entries. */
int cmg_relax_variants(cmg_hierarchy* h, int* inline_out, float* ms_fill, float* ms_inline, int cap, int* n);

/* Mixed precision (no counterpart in the reference, which runs FP64
 * throughout): the loop of AMRMultiGrid::solve with each AMR V-cycle run in
 * FP32 (smoothing, restriction, prolongation, the cycle's own residual
 * updates) on the FP64 residual rounded to FP32, its correction added to the
 * FP64 phi; the composite residual with its flux-register correction, the
 * BiCGStab bottom solve and the norms stay FP64.  Same stopping rules and
 * history as cmg_solve; iterations counts the FP64 refinement steps. */
int cmg_solve_mixed(cmg_hierarchy* h, const cmg_solve_params* p, int zero_phi, int* exit_status, int* iterations,
                    double* history, int history_cap, int* history_len);

/* AMRMultiGrid::computeAMRResidual(phi, rhs, lmax, 0) (AMRMultiGrid.H:738-750). */
int cmg_residual_norm(cmg_hierarchy* h, double* out);

/* TGAHelmOp::setAlphaAndBeta on every operator of the hierarchy, as the
 * reference's heat solvers call it (BackwardEuler::resetAlphaAndBeta,
 * BackwardEuler.cpp:22-31): op 0 scales the coefficients given at creation
 * (AMRPoissonOp.cpp:1103-1108: alpha = a_alpha * alpha0, beta = a_beta *
 * beta0); op 1 takes them as given and recomputes the relaxation coefficient
 * (VCAMRPoissonOp2.cpp:258-318) on every level and multigrid depth. */
int cmg_set_alpha_beta(cmg_hierarchy* h, double alpha, double beta);
/* nsteps backward-Euler steps of the heat equation (BackwardEuler::oneStep,
 * BackwardEuler.cpp:156-189, createEulerRHS :190-226, solveHelm :228-245):
 * phi is the state, the right-hand side set with cmg_set_rhs is the source.
 * Each step forms rhs = a*phi + dt*src (a = 1 for op 0), calls
 * setAlphaAndBeta(1, -dt) and solves (AMRMultiGrid::solve with p) for the new
 * phi from the old one (zero_phi == 0, the heat solvers' choice) or from zero.
 * exit_status and iterations (nsteps entries each, may be NULL) receive each
 * step's solve; the source is left in the right-hand side afterwards. */
int cmg_backward_euler(cmg_hierarchy* h, const cmg_solve_params* p, double dt, int nsteps, int zero_phi,
                       int* exit_status, int* iterations);
/* nsteps steps of the second-order TGA heat solver (AMRTGA<T>::oneStep,
 * AMRTGA.H:420-560): per step the source term (a I + mu4 dt L) S/a and
 * (a I + mu3 dt L) phi^n through the composite operator
 * (AMRMultiGrid::computeAMROperator), then two Helmholtz solves
 * (setAlphaAndBeta(1, -mu2 dt), then (1, -mu1 dt)) from the old phi, with
 * the mu of AMRTGA::setMu.  phi is the state and the right-hand side the
 * source, as for cmg_backward_euler; exit_status and iterations receive the
 * 2 * nsteps solves in order. */
int cmg_tga(cmg_hierarchy* h, const cmg_solve_params* p, double dt, int nsteps, int* exit_status,
            int* iterations);

/* BiCGStab over the whole hierarchy, preconditioned by AMR multigrid: the
 * solve path of the reference's variable-coefficient example
 * (BiCGStabSolver<Vector<LevelData<FArrayBox>*>>::solve, BiCGStabSolver.H:
 * 199-515, over MultilevelLinearOp<FArrayBox>, MultilevelLinearOpI.H, set up
 * as VCPoissonSolve.cpp:146-183 with the max norm).  Each preconditioner call
 * runs mg_iters rounds of (homogeneous residual, one AMR V-cycle with
 * mg_smooth pre, post and bottom smoothings from a zero correction,
 * increment); dot products follow the reference's summation order (each box
 * in k, j, i order, boxes in layout order, levels scaled by dx^3 and summed
 * coarse to fine).  exit_status is the solver's m_exitStatus (1 converged,
 * 2 rho = 0, 3 stalled after num_restarts restarts, -1 iteration limit),
 * iterations its m_iter; history receives the residual norm after every
 * iteration.  Starts from phi as it is, or from zero when zero_phi != 0. */
typedef struct cmg_mlsolve_params {
  int mg_iters, mg_smooth, imax, num_restarts;
  double eps, reps, hang, small;
} cmg_mlsolve_params;
int cmg_solve_multilevel_bicgstab(cmg_hierarchy* h, const cmg_mlsolve_params* p, int zero_phi, int* exit_status,
                                  int* iterations, double* initial_residual, double* final_residual, double* history,
                                  int history_cap, int* history_len);

/* Coarse-to-fine interpolation of a new level, FineInterp::interpToFine
 * (AMRTools/FineInterp.cpp:106-160; FineInterp.H:158-162) with the default
 * PCInterp boundary limiting, refinement ratio 2, one component: every valid
 * cell of phi on `level` (1..finest) from phi on level - 1.  Coarse cells of
 * the layer next to the domain boundary interpolate piecewise constant; the
 * others add the limited central slopes.  piecewise_constant != 0 gives
 * pwcinterpToFine (FineInterp.cpp:162-199; FineInterp.H:164-168).
 * CMG_EINVAL when the level is not properly nested (the interpolation reads
 * grow(coarsen(fine box), 1) & domain from the coarse level). */
int cmg_interp_to_fine(cmg_hierarchy* h, int level, int piecewise_constant);

/* FineInterp as a standalone object (FineInterp.H:59-121): define() with the
 * fine layout and fine problem domain (ratio 2, one component), plus the
 * coarse layout the data come on.  Data are valid cells per box in the given
 * box order, x fastest; on_device selects device or host pointers. */
typedef struct cmg_fine_interp cmg_fine_interp;
int cmg_fine_interp_create(const int fine_domain_lo[3], const int fine_domain_hi[3], int nfine, const cmg_box* fine,
                           int ncoarse, const cmg_box* coarse, cmg_fine_interp** out);
int cmg_fine_interp_run(cmg_fine_interp* fi, const double* coarse, double* fine, int on_device,
                        int piecewise_constant);
int cmg_fine_interp_destroy(cmg_fine_interp* fi);
/* Runs later cmg_fine_interp_run calls on `stream` (a cudaStream_t; NULL: the
 * object's own stream), as cmg_set_stream does for a hierarchy.  With
 * on_device != 0 the run reads `coarse` in stream order, so a caller that
 * produced it on another stream must make this stream wait for it first. */
int cmg_fine_interp_set_stream(cmg_fine_interp* fi, void* stream);
/* 1 when the fused one-kernel path runs (every fine box's coarse staging
 * block fits in shared memory), 0 for the gather + interpolate path. */
int cmg_fine_interp_is_fused(const cmg_fine_interp* fi, int* out);

/* Same value as cmg_residual_norm, allocating no memory on success (no
 * counterpart in the reference, which has no such constraint).  For callers
 * that cannot let the library allocate at call time: a process whose memory
 * pool holds all free device memory, or a loop that must not synchronise the
 * device through cudaMalloc/cudaFree.  The reduction scratch is a fixed
 * device array of 4097 doubles per device (CMG_NOALLOC_MAX_BOXES per-box
 * partials plus one running maximum); hierarchies with a level of more than
 * CMG_NOALLOC_MAX_BOXES boxes, or with more than 16 levels, are rejected with
 * CMG_EINVAL.  The first call on a device looks the scratch up with
 * cudaGetSymbolAddress (that device made current); make it before any stream
 * capture begins on the device.  Every call zeroes the running maximum
 * itself.  Calls that overlap in time on one device share the scratch and
 * race: serialise them.  The address found is kept for the process; a
 * caller that resets a device (cudaDeviceReset) calls
 * cmg_residual_norm_noalloc_forget() afterwards, and its next call on that
 * device looks the scratch up again (outside any capture, as a first call). */
#define CMG_NOALLOC_MAX_BOXES 4096
int cmg_residual_norm_noalloc(cmg_hierarchy* h, double* out);
int cmg_residual_norm_noalloc_forget(void);

/* Fills rhs (all levels) and, for op = 1, a and b from the seeded synthetic
 * workload recipe (Gaussian bumps; exp of a random Fourier series), then
 * finalizes the coefficients. */
int cmg_fill_synthetic(cmg_hierarchy* h, uint64_t seed);
/* The same seeded inputs generated on the device, with the coefficient
 * set-up of cmg_finalize_coefficients done there too (no counterpart in the
 * reference): fast set-up for served requests.  Values agree with
 * cmg_fill_synthetic to within the last bits of exp and cos. */
int cmg_fill_synthetic_device(cmg_hierarchy* h, uint64_t seed);

/* domainSplit (BoxTools/BRMeshRefine.cpp:983-1092), all directions. Boxes are
 * returned in layout order. */
int cmg_domain_split(const int domain_lo[3], const int domain_hi[3], int max_box, int block_factor, cmg_box* out,
                     int cap, int* n);

/* Local motion items of a level's exchange copier (Copier::exchangeDefine +
 * trimEdges, BoxTools/Copier.cpp:1464-1516, 142-177): per item
 * from, to, fromRegion(6), toRegion(6).  Returns the item count in *n. */
int cmg_exchange_plan(const cmg_hierarchy* h, int level, int* items14, int cap, int* n);
/* Local motion items of the coarsened-fine to coarse copier of level >= 1
 * (AMRPoissonOp::buildCopier, AMRElliptic/AMRPoissonOp.cpp:474-483). */
int cmg_coarse_fine_plan(const cmg_hierarchy* h, int level, int* items14, int cap, int* n);

/* Host-only variants (no device state): the same plans for a box list given
 * directly, in layout order after sorting. */
int cmg_layout_exchange_plan(const cmg_box* boxes, int nbox, int* items14, int cap, int* n);
/* The exchange plan of a box list on a domain with periodic directions
 * (periodic[d] nonzero): items from the domain's periodic images carry a
 * fromRegion shifted by the domain length against their toRegion
 * (Copier::define over ProblemDomain's shift iterator, BoxTools/Copier.cpp:903-1110). */
int cmg_layout_exchange_plan_periodic(const cmg_box* boxes, int nbox, const cmg_box* domain, const int* periodic,
                                      int* items14, int cap, int* n);
int cmg_layout_coarse_fine_plan(const cmg_box* fine, int nfine, const cmg_box* coarse, int ncoarse, int* items14,
                                int cap, int* n);

/* Grid generation (host only): the box lists of the examples' hierarchy
 * for the seeded synthetic right-hand side.  Level 0 is domainSplit of
 * [0, n0-1]^3 (BRMeshRefine.cpp:983-1092); each pass tags cells with
 * |rhs| > thresh * max|rhs| on every level, grows the tags by one cell and
 * calls MeshRefine::regrid (MeshRefine.cpp:438-729) with Berger-Rigoutsos
 * clustering (BRMeshRefine::makeBoxes, BRMeshRefine.cpp:213-308), buffer 2,
 * refinement ratio 2, adding one level per pass (as
 * releasedExamples/AMRPoisson/execVariableCoefficient/VClocalFuncs.cpp:398-480).
 * nboxes (capacity nlevels) receives the box count per level, boxes (capacity
 * cap, may be NULL to query) the sorted boxes of every level in turn, ntotal
 * their total. */
int cmg_synthetic_hierarchy(int n0, int nlevels, int max_box, int block_factor, double fill_ratio, uint64_t seed,
                            double thresh, int* nlevels_out, int* nboxes, cmg_box* boxes, int cap, int* ntotal);
/* The same hierarchy with the tagging pass of every level (|rhs| at every
 * cell, max-reduction, threshold, one-cell growth; VClocalFuncs.cpp:586-624)
 * run on the current CUDA device; Berger-Rigoutsos stays on the host.  The
 * right-hand side is evaluated with the CUDA math library, whose exp differs
 * from the host's in the last bit at most, so a cell within a few ulps of the
 * threshold could be tagged differently from cmg_synthetic_hierarchy. */
int cmg_synthetic_hierarchy_device(int n0, int nlevels, int max_box, int block_factor, double fill_ratio,
                                   uint64_t seed, double thresh, int* nlevels_out, int* nboxes, cmg_box* boxes,
                                   int cap, int* ntotal);

/* Batching and serving (no counterpart in the reference, which solves one
 * hierarchy per call).  A request is a seeded synthetic problem: the
 * example hierarchy of cmg_synthetic_hierarchy, operator (op as in
 * cmg_hierarchy_create), solver parameters, precision (mixed != 0:
 * cmg_solve_mixed) and CUDA-graph replay.  cmg_serve runs max_inflight
 * workers; each takes the next request in arrival order (released at its
 * arrival time when open_loop != 0, all at once otherwise), generates its
 * grids, waits until the device memory of the admitted hierarchies plus its
 * own estimate fits in hbm_budget bytes (a request whose estimate alone exceeds
 * the budget fails with CMG_ENOMEM), builds the hierarchy on its own
 * stream, solves, reads phi back (hashed into phi_hash) and frees it.  The
 * solves of all admitted requests overlap on the device; requests share no
 * device data, so every result is the same alone and in the mix.  Times are
 * seconds after the start of the run. */
typedef struct cmg_request {
  double arrival;
  int n0, levels, max_box, block_factor;
  double fill_ratio, thresh;
  uint64_t seed;
  int op;
  double alpha, beta;
  cmg_solve_params params;
  int mixed, graphs;
  int device_tags; /* != 0: tag on the device (cmg_synthetic_hierarchy_device) */
  double timeout;  /* seconds after arrival (after the start when open_loop == 0) to finish by; 0: none */
  const volatile int* cancel; /* NULL, or a flag the caller may set from any thread to cancel the request */
  /* Host-side fault injection (tests): a NaN in one cell of the finest
   * right-hand side once the inputs are generated; cancellation after this
   * many iterations (-1: never). */
  int inject_nan_rhs, inject_cancel_after;
} cmg_request;

typedef struct cmg_request_result {
  int exit_status, iterations;
  int error; /* 0, or the request's status: CMG_EINVAL (invalid description), CMG_ENOMEM (the request alone
                exceeds the budget, or an allocation failed), CMG_EDIVERGED (a residual norm became NaN or
                infinite), CMG_ETIMEOUT, CMG_ECANCELLED, CMG_ECUDA / CMG_EINTERNAL; see message */
  double admitted, started, solved, finished, setup_seconds, solve_seconds, r0, rfinal;
  double grid_seconds, build_seconds, fill_seconds; /* parts of setup_seconds */
  int64_t cells;
  uint64_t device_bytes, phi_hash;
  uint64_t estimate_bytes; /* the admission estimate of the request's device memory */
  int batch_size;          /* requests solved together with this one (cmg_serve_batched), itself included */
  char message[160];       /* empty, or what went wrong */
} cmg_request_result;

/* A failing request ends alone: it releases its memory and admission, and
 * every other request runs as if it had not been there.  Cancellation and the
 * time limit are looked at while a request waits for admission and between
 * its solver iterations.  The call itself fails only on invalid arguments
 * (null arrays, max_inflight < 1, a non-positive budget). */
int cmg_serve(const cmg_request* reqs, int n, double hbm_budget, int max_inflight, int open_loop,
              cmg_request_result* out, double* wall_seconds);
/* cmg_serve with V-cycles batched across requests: a request admitted less
 * than batch_window seconds after another of its class (the same problem
 * recipe, operator, precision and solver parameters; tolerances may differ)
 * joins it, and up to max_batch such requests are solved as one forest
 * (cmg_forest_create), each keeping its own tolerance, stopping rule, time
 * limit, cancellation and status; the first waits at most batch_window for
 * the others.  A request without a partner is solved alone, as cmg_serve
 * does.  Each result is the request's own solve, bit for bit. */
int cmg_serve_batched(const cmg_request* reqs, int n, double hbm_budget, int max_inflight, int open_loop,
                      double batch_window, int max_batch, cmg_request_result* out, double* wall_seconds);

/* Algorithmic bytes moved per V-cycle (roofline numerator). */
int cmg_vcycle_bytes(const cmg_hierarchy* h, const cmg_solve_params* p, double* out);

/* Host seconds cmg_hierarchy_create spent building the plans (layouts,
 * exchange, coarse-fine, flux-register and bottom tables) and setting up the
 * device (allocation, uploads); either pointer may be null. */
int cmg_setup_seconds(const cmg_hierarchy* h, double* plans, double* device);
/* Host plan tables of 1 MiB or more take their storage from blocks that are
 * kept, once freed, for later plans (up to min(8 GiB, physical memory / 8)),
 * so a process that creates hierarchy after hierarchy reuses mapped pages.
 * *kept (may be null) receives the bytes held; release != 0 first gives
 * them all back to the system. */
int cmg_host_blocks(int release, size_t* kept);
/* The CUDA stream every call of this hierarchy runs on (cudaStream_t). */
int cmg_get_stream(const cmg_hierarchy* h, void** stream);
/* Streams (no counterpart in the reference, whose calls are synchronous host
 * code).  After cmg_set_stream every later call of this hierarchy issues its
 * device work on `stream` (a cudaStream_t of the current device; NULL goes
 * back to the hierarchy's own stream), in order with what the caller queued
 * on that stream before the call: device-pointer inputs produced on that
 * stream need no synchronisation.  Work already queued on the previous
 * stream is finished first.  Device memory stays on the hierarchy's own
 * stream, so the caller's stream may be destroyed after the hierarchy's last
 * call that used it has returned.  Calls that return results to the host
 * (norms, histories, host arrays) still synchronise the stream before they
 * return. */
int cmg_set_stream(cmg_hierarchy* h, void* stream);

/* Operator-level calls: one virtual of the reference's operator interfaces
 * (AMRLevelOp, AMRElliptic/AMRMultiGrid.H:39-225; MGLevelOp, MultiGrid.H:
 * 116-160; LinearOp, LinearSolver.H:41-137), as AMRPoissonOp and
 * VCAMRPoissonOp2 implement them, on one level of a hierarchy: what a
 * Chombo program's own AMRMultiGrid / MultiGrid / BiCGStabSolver calls when
 * it drives the GPU operators through include/cmg_chombo.H
 * (GpuAMRPoissonOpFactory as an AMRLevelOpFactory).  Same kernels and
 * operation order as cmg_solve.
 *
 * lev >= 0 names AMR level lev; lev < 0 names multigrid depth -lev below
 * level 0 (AMRPoissonOpFactory::MGnewOp, AMRPoissonOp.cpp:1923-1989), for
 * 1 <= -lev <= cmg_op_num_mg_depths.  Arrays are host memory in the ghosted
 * format: every box's FAB grown by one cell, x fastest, boxes in layout
 * order (the memory of a one-component LevelData<FArrayBox> with one ghost
 * layer, box after box); cmg_op_size gives its length.  Inputs are read whole,
 * ghost cells included (a ghost the operator does not refill is read as the
 * caller left it, as in the reference).  Outputs receive their valid cells;
 * their ghost positions are unspecified.  Boundary conditions are the
 * hierarchy's homogeneous Dirichlet, so `homogeneous` changes nothing for
 * them; on levels >= 1 it selects whether residual sets the homogeneous
 * coarse-fine ghosts first (AMRPoissonOp::residual, AMRPoissonOp.cpp:227-238).
 * Every call copies its arguments to the device and back and synchronises. */
int cmg_op_num_mg_depths(const cmg_hierarchy* h, int* out);
int cmg_op_num_boxes(const cmg_hierarchy* h, int lev, int* out);
int cmg_op_get_boxes(const cmg_hierarchy* h, int lev, cmg_box* out, int cap);
int cmg_op_size(const cmg_hierarchy* h, int lev, int64_t* out);
/* Length of a ghosted array over coarsen(level's boxes, 2) (level >= 1): the
 * layout of AMRMultiGrid's m_resC (createCoarsened, AMRPoissonOp.cpp:459-471). */
int cmg_op_coarsened_size(const cmg_hierarchy* h, int level, int64_t* out);
/* LinearOp::residual: lhs = rhs - L(phi) (OPERATORLAPRES / VCCOMPUTERES3D
 * after exchange and boundary values; AMRPoissonOp.cpp:227-297). */
int cmg_op_residual(cmg_hierarchy* h, int lev, double* lhs, const double* phi, const double* rhs, int homogeneous);
/* LinearOp::applyOp: lhs = L(phi) with homogeneous coarse-fine ghosts
 * (AMRPoissonOp.cpp:332-385). */
int cmg_op_apply(cmg_hierarchy* h, int lev, double* lhs, const double* phi, int homogeneous);
/* MGLevelOp::relax: iterations red-black Gauss-Seidel sweeps (levelGSRB,
 * AMRPoissonOp.cpp:600-632, 1216-1281; VCAMRPoissonOp2.cpp:547-626). */
int cmg_op_relax(cmg_hierarchy* h, int lev, double* phi, const double* rhs, int iterations);
/* LinearOp::preCond: cor = res / diagonal, then two sweeps
 * (AMRPoissonOp.cpp:304-329, VCAMRPoissonOp2.cpp:93-127). */
int cmg_op_precond(cmg_hierarchy* h, int lev, double* cor, const double* res);
/* MGLevelOp::restrictResidual: res_coarse (level lev - 1, i.e. the next
 * multigrid depth) = average of rhs - L(phi) (RESTRICTRES(VC3D),
 * AMRPoissonOp.cpp:651-703).  lev <= 0. */
int cmg_op_restrict_residual(cmg_hierarchy* h, int lev, double* res_coarse, const double* phi, const double* rhs);
/* MGLevelOp::prolongIncrement: phi += corr_coarse at the parent cell (PROLONG,
 * AMRPoissonOp.cpp:706-733).  lev <= 0; corr_coarse on level lev - 1. */
int cmg_op_prolong_increment(cmg_hierarchy* h, int lev, double* phi, const double* corr_coarse);
/* The AMROperator / AMRResidual family (AMRPoissonOp.cpp:736-858) on AMR
 * level `level`: inhomogeneous quadratic coarse-fine ghosts from phi_coarse
 * (level - 1) when it is not NULL, exchange and boundary values, then
 *   form 0: out = L(phi), with the flux-register correction from phi_fine
 *           (level + 1) when it is not NULL (AMROperator, AMROperatorNC/NF);
 *   form 1: the same followed by out = rhs - out as axby(out, out, rhs, -1, 1)
 *           (AMRResidual, AMRResidualNC);
 *   form 2: out = rhs - L(phi) in residualI's own expression, phi_fine NULL
 *           (AMRResidualNF).
 * Without phi_coarse the coarse-fine ghosts are phi's own (as the reference's
 * applyOpI leaves them).  On return phi holds the ghost values the operator
 * used (its valid cells unchanged): the reference fills the ghost cells of
 * its const phi argument the same way. */
int cmg_op_amr_operator(cmg_hierarchy* h, int level, int form, double* out, const double* phi_fine,
                        double* phi, const double* phi_coarse, const double* rhs);
/* AMRLevelOp::AMRRestrictS (AMRPoissonOp.cpp:877-919), level >= 1: the
 * residual of `correction` against `residual` with coarse-fine ghosts from
 * coarse_correction (level - 1), averaged onto the coarsened-fine layout
 * (res_coarsened, cmg_op_coarsened_size doubles).  correction == NULL is
 * a_skip_res: `residual` itself is averaged (the FAS restriction). */
int cmg_op_amr_restrict(cmg_hierarchy* h, int level, double* res_coarsened, const double* residual,
                        const double* correction, const double* coarse_correction);
/* assignCopier(coarse, coarsened, m_resCopier) of AMRMultiGrid::AMRVCycle
 * (AMRMultiGrid.H:1391): the valid cells of level - 1 under level take the
 * coarsened-fine values; coarse (level - 1) is read and written. */
int cmg_op_assign_coarsened(cmg_hierarchy* h, int level, double* coarse, const double* coarsened);
/* AMRLevelOp::AMRProlongS / AMRProlong (AMRPoissonOp.cpp:926-990), level >= 1:
 * correction += coarse_correction (level - 1) at the parent cell. */
int cmg_op_amr_prolong(cmg_hierarchy* h, int level, double* correction, const double* coarse_correction);
/* AMRLevelOp::AMRUpdateResidual (AMRPoissonOp.cpp:1045-1054), level >= 1:
 * residual -= L(correction) with coarse-fine ghosts from coarse_correction. */
int cmg_op_amr_update_residual(cmg_hierarchy* h, int level, double* residual, const double* correction,
                               const double* coarse_correction);
/* QuadCFInterp::coarseFineInterp (AMRTools/QuadCFInterp.cpp:845-889), level
 * >= 1: the coarse-fine face ghosts of phi from phi_coarse (level - 1), by the
 * tangential Taylor expansion of the coarse data (PHISTAR, QuadCFStencil) and
 * the quadratic through it and two fine cells (QUADINTERP / interpOnIVS).
 * phi is read whole and returned whole: valid cells unchanged, coarse-fine
 * ghosts set, every other ghost as it was. */
int cmg_op_cf_interp(cmg_hierarchy* h, int level, double* phi, const double* phi_coarse);
/* AMRLevelOp::zeroCovered (AMRMultiGrid.H:197-201): zero the valid cells of
 * `level` covered by level + 1. */
int cmg_op_zero_covered(cmg_hierarchy* h, int level, double* data);
/* LevelDataOps (AMRElliptic/LevelDataOps.H:179-281): lhs = a x + b y
 * (x*a then + y*b), lhs += scale x, lhs *= scale. */
int cmg_op_axby(cmg_hierarchy* h, int lev, double* lhs, const double* x, const double* y, double a, double b);
int cmg_op_incr(cmg_hierarchy* h, int lev, double* lhs, const double* x, double scale);
int cmg_op_scale(cmg_hierarchy* h, int lev, double* lhs, double scale);
/* LevelDataOps::dotProduct (LevelDataOps.H:109-131): per box in k, j, i
 * order, boxes summed in layout order. */
int cmg_op_dot(cmg_hierarchy* h, int lev, const double* x, const double* y, double* out);
/* norm(LevelData, ord) as AMRPoissonOp::norm computes it (BoxTools/
 * BoxLayoutData.cpp:23-93, FArrayBox::norm/sumPow): ord 0 the max norm (a NaN
 * anywhere gives NaN), 1 the sum of |x|, 2 the 2-norm, each box in pencil
 * order. */
int cmg_op_norm(cmg_hierarchy* h, int lev, const double* x, int ord, double* out);

/* Kernel-class device timing, the counterpart of the reference's CH_TIMER
 * trace timers (BaseTools/CH_Timer.H:44-163): while enabled, every launch of a
 * class is bracketed by CUDA events on the hierarchy's stream.  Classes:
 * 0 = red-black relaxation on the finest AMR level, 1 = residual / operator
 * application, 2 = ghost fills (exchange, boundary and homogeneous coarse-fine
 * values), 3 = bottom solves, 4 = red-black relaxation on every other level,
 * 5 = fine interpolation (cmg_interp_to_fine).
 * cmg_profile_read returns launches, total device milliseconds and the
 * algorithmic bytes of those launches since the last enable. */
int cmg_profile_enable(cmg_hierarchy* h, int on);
/* Total kernel launches issued by this library in this process. */
int cmg_launch_count(int64_t* out);
int cmg_profile_read(cmg_hierarchy* h, int kernel_class, int64_t* launches, double* ms, double* bytes);

#ifdef __cplusplus
}
#endif

#endif
