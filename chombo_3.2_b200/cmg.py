"""ctypes binding of libcmg.so (include/cmg.h) for the tests and the benchmark.

The library is the product; this module only marshals numpy arrays and
raises on any non-zero status.  It fails loudly when libcmg.so is missing:
there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcmg.so")


class CmgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cmg status {code}: {msg}")
        self.code = code


class Box(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3)]


# Status codes (cmg.h).
CMG_OK, CMG_EINVAL, CMG_ENOMEM, CMG_ECUDA, CMG_EINTERNAL, CMG_EDIVERGED, CMG_ETIMEOUT, CMG_ECANCELLED = range(8)
# Homogeneous boundary types of a domain face (cmg_hierarchy_create_bc).
BC_DIRICHLET, BC_NEUMANN, BC_PERIODIC = 0, 1, 2


class SolveParams(ctypes.Structure):
    _fields_ = [("pre", ctypes.c_int), ("post", ctypes.c_int), ("bottom", ctypes.c_int),
                ("num_mg", ctypes.c_int), ("iter_max", ctypes.c_int), ("imin", ctypes.c_int),
                ("eps", ctypes.c_double), ("hang", ctypes.c_double), ("norm_thresh", ctypes.c_double),
                ("iter_min", ctypes.c_int)]


class MLSolveParams(ctypes.Structure):
    _fields_ = [("mg_iters", ctypes.c_int), ("mg_smooth", ctypes.c_int), ("imax", ctypes.c_int),
                ("num_restarts", ctypes.c_int), ("eps", ctypes.c_double), ("reps", ctypes.c_double),
                ("hang", ctypes.c_double), ("small", ctypes.c_double)]


def mlsolve_params(mg_iters=1, mg_smooth=4, imax=80, num_restarts=5, eps=1e-6, reps=1e-12, hang=1e-8, small=1e-30):
    """Parameters of cmg_solve_multilevel_bicgstab; defaults are the reference's MultilevelLinearOp and
    BiCGStabSolver defaults."""
    return MLSolveParams(mg_iters, mg_smooth, imax, num_restarts, eps, reps, hang, small)


def solve_params(pre=4, post=4, bottom=4, num_mg=1, iter_max=100, imin=5, eps=1e-10, hang=1e-10,
                 norm_thresh=1e-30, iter_min=-1):
    return SolveParams(pre, post, bottom, num_mg, iter_max, imin, eps, hang, norm_thresh, iter_min)


class BottomParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("imax", ctypes.c_int), ("num_restarts", ctypes.c_int),
                ("norm_type", ctypes.c_int), ("eps", ctypes.c_double), ("hang", ctypes.c_double),
                ("small", ctypes.c_double)]


class Request(ctypes.Structure):
    _fields_ = [("arrival", ctypes.c_double), ("n0", ctypes.c_int), ("levels", ctypes.c_int),
                ("max_box", ctypes.c_int), ("block_factor", ctypes.c_int), ("fill_ratio", ctypes.c_double),
                ("thresh", ctypes.c_double), ("seed", ctypes.c_uint64), ("op", ctypes.c_int),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("params", SolveParams),
                ("mixed", ctypes.c_int), ("graphs", ctypes.c_int), ("device_tags", ctypes.c_int),
                ("timeout", ctypes.c_double), ("cancel", ctypes.POINTER(ctypes.c_int)),
                ("inject_nan_rhs", ctypes.c_int), ("inject_cancel_after", ctypes.c_int)]


class RequestResult(ctypes.Structure):
    _fields_ = [("exit_status", ctypes.c_int), ("iterations", ctypes.c_int), ("error", ctypes.c_int),
                ("admitted", ctypes.c_double), ("started", ctypes.c_double), ("solved", ctypes.c_double),
                ("finished", ctypes.c_double), ("setup_seconds", ctypes.c_double),
                ("solve_seconds", ctypes.c_double), ("r0", ctypes.c_double), ("rfinal", ctypes.c_double),
                ("grid_seconds", ctypes.c_double), ("build_seconds", ctypes.c_double),
                ("fill_seconds", ctypes.c_double),
                ("cells", ctypes.c_int64), ("device_bytes", ctypes.c_uint64), ("phi_hash", ctypes.c_uint64),
                ("estimate_bytes", ctypes.c_uint64), ("batch_size", ctypes.c_int), ("message", ctypes.c_char * 160)]


def host_blocks(release=False):
    """Bytes of freed host plan-table blocks kept for reuse by later plans; release=True gives them back first."""
    kept = ctypes.c_size_t()
    _check(lib().cmg_host_blocks(1 if release else 0, ctypes.byref(kept)))
    return kept.value


def serve(requests, hbm_budget=120e9, max_inflight=16, open_loop=True, batch_window=0.0, max_batch=16):
    """Runs cmg_serve over a list of dicts with Request fields; returns (results, wall seconds).  batch_window > 0:
    cmg_serve_batched, requests of one class in flight together solved as one forest."""
    n = len(requests)
    arr = (Request * max(n, 1))()
    for i, r in enumerate(requests):
        q = arr[i]
        q.arrival = r.get("arrival", 0.0)
        q.n0, q.levels = r["n0"], r.get("levels", 1)
        q.max_box, q.block_factor = r.get("max_box", 32), r.get("block_factor", 8)
        q.fill_ratio, q.thresh = r.get("fill_ratio", 0.75), r.get("thresh", 0.1)
        q.seed, q.op = r.get("seed", 20261203), r.get("op", 0)
        q.alpha, q.beta = r.get("alpha", 0.0), r.get("beta", 1.0)
        q.params = r.get("params") or solve_params(eps=r.get("eps", 1e-10))
        q.mixed, q.graphs = int(r.get("mixed", True)), int(r.get("graphs", True))
        q.device_tags = int(r.get("device_tags", False))
        q.timeout = r.get("timeout", 0.0)
        if r.get("cancel") is not None:  # a ctypes.c_int the caller may set while the call runs
            q.cancel = ctypes.pointer(r["cancel"])
        q.inject_nan_rhs = int(r.get("inject_nan_rhs", False))
        q.inject_cancel_after = int(r.get("inject_cancel_after", -1))
    out = (RequestResult * max(n, 1))()
    wall = ctypes.c_double()
    if batch_window > 0:
        _check(lib().cmg_serve_batched(arr, n, ctypes.c_double(hbm_budget), int(max_inflight), int(open_loop),
                                       ctypes.c_double(batch_window), int(max_batch), out, ctypes.byref(wall)))
    else:
        _check(lib().cmg_serve(arr, n, ctypes.c_double(hbm_budget), int(max_inflight), int(open_loop), out,
                               ctypes.byref(wall)))
    keys = [f[0] for f in RequestResult._fields_]
    res = [{k: getattr(out[i], k) for k in keys} for i in range(n)]
    for r in res:
        r["message"] = r["message"].decode(errors="replace")
    return res, wall.value


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} not built: run `make -C chombo_3.2_b200`")
        L = ctypes.CDLL(LIB_PATH)
        L.cmg_last_error.restype = ctypes.c_char_p
        L.cmg_fill_synthetic.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        _lib = L
    return _lib


def _check(rc):
    if rc != CMG_OK:
        raise CmgError(rc, lib().cmg_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def boxes_array(boxes):
    arr = (Box * len(boxes))()
    for i, b in enumerate(boxes):
        arr[i].lo[:] = list(b[0:3])
        arr[i].hi[:] = list(b[3:6])
    return arr


def synthetic_hierarchy(n0, levels, max_box=32, block_factor=8, fill_ratio=0.75, seed=20261203, thresh=0.1,
                        device_tags=False):
    """Box lists (lo0, lo1, lo2, hi0, hi1, hi2) per level of the seeded example hierarchy; device_tags runs the
    tagging passes on the current CUDA device (cmg_synthetic_hierarchy_device)."""
    L = lib()
    fn = L.cmg_synthetic_hierarchy_device if device_tags else L.cmg_synthetic_hierarchy
    nl, tot = ctypes.c_int(), ctypes.c_int()
    counts = (ctypes.c_int * levels)()
    args = (int(n0), int(levels), int(max_box), int(block_factor), ctypes.c_double(fill_ratio),
            ctypes.c_uint64(seed), ctypes.c_double(thresh), ctypes.byref(nl), counts)
    cap = 1 << 16
    out = (Box * cap)()
    _check(fn(*args, out, cap, ctypes.byref(tot)))
    if tot.value > cap:
        out = (Box * tot.value)()
        _check(fn(*args, out, tot.value, ctypes.byref(tot)))
    res, k = [], 0
    for l in range(nl.value):
        res.append([tuple(out[k + i].lo) + tuple(out[k + i].hi) for i in range(counts[l])])
        k += counts[l]
    return res


def domain_split(lo, hi, max_box, block_factor):
    L = lib()
    n = ctypes.c_int()
    _check(L.cmg_domain_split((ctypes.c_int * 3)(*lo), (ctypes.c_int * 3)(*hi), max_box, block_factor, None, 0,
                              ctypes.byref(n)))
    out = (Box * n.value)()
    _check(L.cmg_domain_split((ctypes.c_int * 3)(*lo), (ctypes.c_int * 3)(*hi), max_box, block_factor, out,
                              n.value, ctypes.byref(n)))
    return [tuple(b.lo) + tuple(b.hi) for b in out]


def launch_count():
    n = ctypes.c_int64()
    _check(lib().cmg_launch_count(ctypes.byref(n)))
    return n.value


def _plan(fn, *args):
    n = ctypes.c_int()
    _check(fn(*args, None, 0, ctypes.byref(n)))
    buf = np.zeros(14 * max(n.value, 1), dtype=np.int32)
    _check(fn(*args, _ptr(buf), n.value, ctypes.byref(n)))
    return buf[:14 * n.value].reshape(n.value, 14)


def layout_exchange_plan(boxes):
    arr = boxes_array(boxes)
    return _plan(lib().cmg_layout_exchange_plan, arr, len(boxes))


def layout_exchange_plan_periodic(boxes, domain, periodic):
    """Exchange plan on ``domain`` (lo, hi) with the directions in ``periodic``
    (three flags) wrapping around."""
    arr = boxes_array(boxes)
    dom = boxes_array([tuple(domain)])
    per = np.asarray([1 if p else 0 for p in periodic], dtype=np.int32)
    return _plan(lib().cmg_layout_exchange_plan_periodic, arr, len(boxes), dom, _ptr(per))


def layout_coarse_fine_plan(fine, coarse):
    fa, ca = boxes_array(fine), boxes_array(coarse)
    return _plan(lib().cmg_layout_coarse_fine_plan, fa, len(fine), ca, len(coarse))


class FineInterp:
    """FineInterp (AMRTools/FineInterp.H) as a standalone object
    (cmg_fine_interp_*): fine layout and fine problem domain, refinement ratio
    2, and the coarse layout the data come on.  interp_to_fine takes the
    coarse level's valid cells (per box in order, x fastest) and returns the
    fine level's."""

    def __init__(self, fine_domain, fine_boxes, coarse_boxes):
        lo, hi = fine_domain[0:3], fine_domain[3:6]
        h = ctypes.c_void_p()
        _check(lib().cmg_fine_interp_create((ctypes.c_int * 3)(*lo), (ctypes.c_int * 3)(*hi), len(fine_boxes),
                                            boxes_array(fine_boxes), len(coarse_boxes), boxes_array(coarse_boxes),
                                            ctypes.byref(h)))
        self.h = h
        self.nfine = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in fine_boxes)
        self.ncoarse = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in coarse_boxes)

    def interp_to_fine(self, coarse, pwc=False, out=None):
        """Host arrays in and out; out (float64, nfine cells, contiguous) is filled and returned when given,
        else a new array."""
        a = np.ascontiguousarray(coarse, dtype=np.float64)
        if a.size != self.ncoarse:
            raise ValueError(f"coarse data has {a.size} cells, the coarse layout {self.ncoarse}")
        if out is None:
            out = np.empty(self.nfine, dtype=np.float64)
        elif out.dtype != np.float64 or out.size != self.nfine or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a contiguous float64 array of {self.nfine} cells")
        _check(lib().cmg_fine_interp_run(self.h, _ptr(a), _ptr(out), 0, int(pwc)))
        return out

    def interp_to_fine_device(self, coarse_ptr, fine_ptr, pwc=False):
        """The same from and into device memory (cmg_fine_interp_run with on_device=1), in the order of the
        object's stream (set_stream)."""
        _check(lib().cmg_fine_interp_run(self.h, ctypes.c_void_p(coarse_ptr), ctypes.c_void_p(fine_ptr), 1,
                                         int(pwc)))

    def set_stream(self, stream):
        """Runs later interpolations on `stream` (a cudaStream_t as an int; 0/None: the object's own)."""
        _check(lib().cmg_fine_interp_set_stream(self.h, ctypes.c_void_p(stream or None)))

    def is_fused(self):
        out = ctypes.c_int()
        _check(lib().cmg_fine_interp_is_fused(self.h, ctypes.byref(out)))
        return bool(out.value)

    def close(self):
        if self.h:
            _check(lib().cmg_fine_interp_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Hierarchy:
    """One AMR hierarchy with device-resident state (cmg_hierarchy)."""

    def __init__(self, n0, level_boxes, op=0, alpha=0.0, beta=1.0, dx0=None, bc=None):
        """bc: None (homogeneous Dirichlet on every face) or six face types, x-lo, x-hi, y-lo, y-hi, z-lo, z-hi,
        each BC_DIRICHLET / BC_NEUMANN / BC_PERIODIC or the letters 'D' / 'N' / 'P' (a string such as "NNNNND";
        periodic directions on both faces, one-level hierarchies)."""
        L = lib()
        self.nlev = len(level_boxes)
        counts = (ctypes.c_int * self.nlev)(*[len(b) for b in level_boxes])
        flat = [b for lev in level_boxes for b in lev]
        arr = boxes_array(flat)
        h = ctypes.c_void_p()
        dx0 = 1.0 / n0 if dx0 is None else dx0
        bcs = None
        if bc is not None:
            letters = {"D": BC_DIRICHLET, "N": BC_NEUMANN, "P": BC_PERIODIC}
            codes = [letters.get(x, x) if isinstance(x, str) else int(x) for x in bc]
            if len(codes) != 6:
                raise ValueError("bc needs six face types")
            bcs = (ctypes.c_int * 6)(*codes)
        _check(L.cmg_hierarchy_create_bc((ctypes.c_int * 3)(0, 0, 0), (ctypes.c_int * 3)(n0 - 1, n0 - 1, n0 - 1),
                                         ctypes.c_double(dx0), self.nlev, counts, arr, op, ctypes.c_double(alpha),
                                         ctypes.c_double(beta), bcs, ctypes.byref(h)))
        self.h = h
        self.op = op

    def close(self):
        if self.h:
            _check(lib().cmg_hierarchy_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def num_cells(self, level):
        n = ctypes.c_int64()
        _check(lib().cmg_num_cells(self.h, level, ctypes.byref(n)))
        return n.value

    def num_faces(self, level, d):
        n = ctypes.c_int64()
        _check(lib().cmg_num_faces(self.h, level, d, ctypes.byref(n)))
        return n.value

    def boxes(self, level):
        n = ctypes.c_int()
        _check(lib().cmg_num_boxes(self.h, level, ctypes.byref(n)))
        out = (Box * n.value)()
        _check(lib().cmg_get_boxes(self.h, level, out, n.value))
        return [tuple(b.lo) + tuple(b.hi) for b in out]

    def fill_synthetic(self, seed, device=False):
        fn = lib().cmg_fill_synthetic_device if device else lib().cmg_fill_synthetic
        _check(fn(self.h, ctypes.c_uint64(seed)))

    def set_rhs(self, level, data):
        a = np.ascontiguousarray(data, dtype=np.float64)
        _check(lib().cmg_set_rhs(self.h, level, _ptr(a), 0))

    def set_acoef(self, level, data):
        a = np.ascontiguousarray(data, dtype=np.float64)
        _check(lib().cmg_set_acoef(self.h, level, _ptr(a), 0))

    def set_bcoef(self, level, d, data):
        a = np.ascontiguousarray(data, dtype=np.float64)
        _check(lib().cmg_set_bcoef(self.h, level, d, _ptr(a), 0))

    def finalize_coefficients(self):
        _check(lib().cmg_finalize_coefficients(self.h))

    def phi(self, level):
        out = np.empty(self.num_cells(level), dtype=np.float64)
        _check(lib().cmg_get_phi(self.h, level, _ptr(out), 0))
        return out

    def get_rhs(self, level):
        out = np.empty(self.num_cells(level), dtype=np.float64)
        _check(lib().cmg_get_rhs(self.h, level, _ptr(out), 0))
        return out

    def set_phi(self, level, data):
        a = np.ascontiguousarray(data, dtype=np.float64)
        _check(lib().cmg_set_phi(self.h, level, _ptr(a), 0))

    def solve(self, params=None, zero_phi=True, mixed=False):
        """AMRMultiGrid::solve on the device; mixed=True runs the FP32
        V-cycles inside FP64 iterative refinement (cmg_solve_mixed)."""
        p = params or solve_params()
        hist = np.zeros(max(p.iter_max, p.iter_min) + 2, dtype=np.float64)
        st, it, hl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        fn = lib().cmg_solve_mixed if mixed else lib().cmg_solve
        rc = fn(self.h, ctypes.byref(p), int(zero_phi), ctypes.byref(st), ctypes.byref(it),
                _ptr(hist), len(hist), ctypes.byref(hl))
        if rc != CMG_EDIVERGED:
            _check(rc)
        return {"exit_status": st.value, "iterations": it.value, "history": hist[:min(hl.value, len(hist))].copy(),
                "diverged": rc == CMG_EDIVERGED}

    def set_alpha_beta(self, alpha, beta):
        """TGAHelmOp::setAlphaAndBeta on every operator of the hierarchy (cmg_set_alpha_beta)."""
        _check(lib().cmg_set_alpha_beta(self.h, ctypes.c_double(alpha), ctypes.c_double(beta)))

    def interp_to_fine(self, level, pwc=False):
        """FineInterp::interpToFine (pwc: pwcinterpToFine) of phi: every valid
        cell of `level` from phi on level - 1 (cmg_interp_to_fine)."""
        _check(lib().cmg_interp_to_fine(self.h, level, int(pwc)))

    def backward_euler(self, params, dt, nsteps, zero_phi=False):
        """nsteps BackwardEuler::oneStep steps on phi with the right-hand side as the source
        (cmg_backward_euler); returns each step's exit status and iteration count."""
        st = (ctypes.c_int * max(nsteps, 1))()
        it = (ctypes.c_int * max(nsteps, 1))()
        _check(lib().cmg_backward_euler(self.h, ctypes.byref(params), ctypes.c_double(dt), int(nsteps),
                                        int(zero_phi), st, it))
        return [{"exit_status": st[n], "iterations": it[n]} for n in range(nsteps)]

    def tga(self, params, dt, nsteps):
        """nsteps AMRTGA::oneStep steps on phi with the right-hand side as the source (cmg_tga); returns the
        2 * nsteps Helmholtz solves' exit status and iteration count."""
        n = 2 * nsteps
        st = (ctypes.c_int * max(n, 1))()
        it = (ctypes.c_int * max(n, 1))()
        _check(lib().cmg_tga(self.h, ctypes.byref(params), ctypes.c_double(dt), int(nsteps), st, it))
        return [{"exit_status": st[k], "iterations": it[k]} for k in range(n)]

    def solve_bicgstab(self, params=None, zero_phi=True):
        """BiCGStab over MultilevelLinearOp preconditioned by AMR multigrid (cmg_solve_multilevel_bicgstab)."""
        p = params or mlsolve_params()
        hist = np.zeros(p.imax + 1, dtype=np.float64)
        st, it, hl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        r0, rf = ctypes.c_double(), ctypes.c_double()
        _check(lib().cmg_solve_multilevel_bicgstab(self.h, ctypes.byref(p), int(zero_phi), ctypes.byref(st),
                                                   ctypes.byref(it), ctypes.byref(r0), ctypes.byref(rf), _ptr(hist),
                                                   len(hist), ctypes.byref(hl)))
        return {"exit_status": st.value, "iterations": it.value, "initial_residual": r0.value,
                "final_residual": rf.value, "history": hist[:hl.value].copy()}

    def set_relax_mode(self, mode):
        _check(lib().cmg_set_relax_mode(self.h, int(mode)))

    def setup_seconds(self):
        """(plan building, device set-up) host seconds of the hierarchy's creation."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(lib().cmg_setup_seconds(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_bottom_solver(self, kind=0, imax=None, num_restarts=5, norm_type=2, eps=1e-6, hang=None, small=1e-30):
        """kind 0 BiCGStabSolver (defaults imax 80, hang 1e-8), 1 RelaxSolver (defaults imax 40, hang 0)."""
        if imax is None:
            imax = 80 if kind == 0 else 40
        if hang is None:
            hang = 1e-8 if kind == 0 else 0.0
        p = BottomParams(int(kind), int(imax), int(num_restarts), int(norm_type), float(eps), float(hang),
                         float(small))
        _check(lib().cmg_set_bottom_solver(self.h, ctypes.byref(p)))

    def set_bottom_grid(self, mode):
        """-1 automatic, 0 one block per hierarchy, 1 the whole device; returns whether the grid-wide bottom
        solve is in use."""
        on = ctypes.c_int()
        _check(lib().cmg_set_bottom_grid(self.h, int(mode), ctypes.byref(on)))
        return bool(on.value)

    def relax_variants(self):
        n = ctypes.c_int()
        _check(lib().cmg_relax_variants(self.h, None, None, None, 0, ctypes.byref(n)))
        v = (ctypes.c_int * max(n.value, 1))()
        a = (ctypes.c_float * max(n.value, 1))()
        b = (ctypes.c_float * max(n.value, 1))()
        _check(lib().cmg_relax_variants(self.h, v, a, b, n.value, ctypes.byref(n)))
        names = {0: "fill", 1: "in-pass ghosts", 2: "one-block sweeps", 3: "fused sweeps"}
        return [{"variant": names.get(v[i], v[i]), "ms_fill": a[i], "ms_best_other": b[i]} for i in range(n.value)]

    def use_graphs(self, on=True):
        _check(lib().cmg_use_graphs(self.h, int(on)))

    def residual_norm(self):
        r = ctypes.c_double()
        _check(lib().cmg_residual_norm(self.h, ctypes.byref(r)))
        return r.value

    def residual_norm_noalloc(self):
        r = ctypes.c_double()
        _check(lib().cmg_residual_norm_noalloc(self.h, ctypes.byref(r)))
        return r.value

    def stream(self):
        s = ctypes.c_void_p()
        _check(lib().cmg_get_stream(self.h, ctypes.byref(s)))
        return s.value

    def profile_enable(self, on=True):
        _check(lib().cmg_profile_enable(self.h, int(on)))

    def profile_read(self, kernel_class):
        n, ms, b = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        _check(lib().cmg_profile_read(self.h, kernel_class, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(b)))
        return n.value, ms.value, b.value

    def set_rhs_ptr(self, level, ptr, on_device):
        _check(lib().cmg_set_rhs(self.h, level, ctypes.c_void_p(ptr), int(on_device)))

    def get_rhs_ptr(self, level, ptr, on_device):
        _check(lib().cmg_get_rhs(self.h, level, ctypes.c_void_p(ptr), int(on_device)))

    def get_phi_ptr(self, level, ptr, on_device):
        _check(lib().cmg_get_phi(self.h, level, ctypes.c_void_p(ptr), int(on_device)))

    def vcycle_bytes(self, params=None):
        p = params or solve_params()
        r = ctypes.c_double()
        _check(lib().cmg_vcycle_bytes(self.h, ctypes.byref(p), ctypes.byref(r)))
        return r.value


class Forest(Hierarchy):
    """A forest (cmg_forest_create): several hierarchies with the same n0, level count, operator and boundary
    types, whose level-0 layouts coarsen alike, solved together (one launch per V-cycle operation for all of
    them).  `hierarchies` is a list of per-hierarchy level box lists.  Level data is the hierarchies' data one
    after the other; phi(k, level) and set_rhs(k, level, data) address one hierarchy."""

    def __init__(self, n0, hierarchies, op=0, alpha=0.0, beta=1.0, dx0=None, bc=None):
        L = lib()
        self.nh = len(hierarchies)
        self.nlev = len(hierarchies[0])
        counts = [len(lev) for hb in hierarchies for lev in hb]
        if len(counts) != self.nh * self.nlev:
            raise ValueError("every hierarchy of a forest has the same number of levels")
        arr = boxes_array([b for hb in hierarchies for lev in hb for b in lev])
        bcs = None
        if bc is not None:
            bcs = (ctypes.c_int * 6)(*[{"D": BC_DIRICHLET, "N": BC_NEUMANN, "P": BC_PERIODIC}.get(x, x) if isinstance(x, str)
                                       else int(x) for x in bc])
        h = ctypes.c_void_p()
        dx0 = 1.0 / n0 if dx0 is None else dx0
        _check(L.cmg_forest_create(self.nh, (ctypes.c_int * 3)(0, 0, 0), (ctypes.c_int * 3)(n0 - 1, n0 - 1, n0 - 1),
                                   ctypes.c_double(dx0), self.nlev, (ctypes.c_int * len(counts))(*counts), arr, op,
                                   ctypes.c_double(alpha), ctypes.c_double(beta), bcs, ctypes.byref(h)))
        self.h = h
        self.op = op

    def cells(self, k, level):
        n = ctypes.c_int64()
        _check(lib().cmg_forest_cells(self.h, k, level, ctypes.byref(n)))
        return n.value

    def _slice(self, k, level):
        a = sum(self.cells(j, level) for j in range(k))
        return slice(a, a + self.cells(k, level))

    def fill_synthetic(self, seeds, device=True):
        """The device generator of every hierarchy with its own seed (cmg_forest_fill_synthetic)."""
        if not device:
            raise ValueError("a forest fills its synthetic inputs on the device")
        arr = (ctypes.c_uint64 * self.nh)(*seeds)
        _check(lib().cmg_forest_fill_synthetic(self.h, arr))

    def phi(self, k, level):
        return Hierarchy.phi(self, level)[self._slice(k, level)].copy()

    def set_rhs(self, k, level, data):
        full = self.get_rhs(level)
        full[self._slice(k, level)] = np.asarray(data, dtype=np.float64)
        Hierarchy.set_rhs(self, level, full)

    def solve(self, params=None, zero_phi=True, mixed=False):
        """Every hierarchy's AMRMultiGrid solve at once (cmg_forest_solve): a list of per-hierarchy results."""
        p = params or solve_params()
        st = (ctypes.c_int * self.nh)()
        it = (ctypes.c_int * self.nh)()
        fn = (ctypes.c_double * self.nh)()
        rc = lib().cmg_forest_solve(self.h, ctypes.byref(p), int(zero_phi), int(mixed), st, it, fn)
        if rc != CMG_EDIVERGED:
            _check(rc)
        return [{"exit_status": st[k], "iterations": it[k], "final_norm": fn[k], "diverged": rc == CMG_EDIVERGED}
                for k in range(self.nh)]
