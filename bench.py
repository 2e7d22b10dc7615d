#!/usr/bin/env python
"""Benchmark of the AMR multigrid solve (AMRMultiGrid::solve over
VCAMRPoissonOp2) on the 3-level variable-coefficient Helmholtz hierarchy:
base 128^3, refinement ratio 2, blocking factor 8, max box 32, fill ratio 0.75,
alpha = 1, beta = -1, coefficients exp of a seeded Fourier series in
[0.1, 10], seeded Gaussian-bump right-hand side, homogeneous Dirichlet,
4 + 4 red-black smooths, BiCGStab bottom, zero initial guess to a 1e-10
relative residual.  One step = one full solve.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0).  Under torchrun every rank solves its own
replica of the hierarchy (independent solves shard with no collective);
timing is the max over ranks.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle")
MLORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_mlbicgstab")
FIORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_fineinterp")
OMPORACLE = os.path.join(ROOT, "oracle", "_ref", "omp", "cmg_oracle")
PROFILE_CLASSES = ["relax_finest", "residual_op", "ghost_fill", "bottom", "relax_other"]
METRIC = "Poisson solves/s & p50/p99 latency at 1e-10 rel. residual; V-cycle HBM GB/s"
WORKLOADS = {
    "config1": {
        "golden": "config1_vc_3lev_128",
        "name": "3-level VC Helmholtz (VCAMRPoissonOp2 alpha=1 beta=-1), base 128^3, ratio 2, block 8, "
                "max box 32, fill 0.75, Dirichlet, GSRB 4+4, BiCGStab bottom, rel. residual 1e-10",
    },
    "config2": {
        "golden": "config2_vc_3lev_256",
        "mixed": True,
        "name": "3-level VC Helmholtz (VCAMRPoissonOp2 alpha=1 beta=-1), base 256^3, ratio 2, block 8, "
                "max box 32, fill 0.75, Dirichlet, GSRB 4+4, BiCGStab bottom, rel. residual 1e-10; FP32 "
                "V-cycles inside FP64 iterative refinement (residual, reflux, bottom, norms FP64)",
    },
    "config2-fp64": {
        "golden": "config2_vc_3lev_256",
        "name": "3-level VC Helmholtz (VCAMRPoissonOp2 alpha=1 beta=-1), base 256^3, ratio 2, block 8, "
                "max box 32, fill 0.75, Dirichlet, GSRB 4+4, BiCGStab bottom, rel. residual 1e-10; plain FP64",
    },
    "config1-bicgstab": {
        "golden": "config1_vc_3lev_128",
        "solver": "bicgstab",
        "bicgstab": {"mg_iters": 2, "mg_smooth": 4, "eps": 1e-10, "imax": 100},
        "name": "3-level VC Helmholtz, base 128^3 (as config1), solved as the variable-coefficient example solves: "
                "BiCGStab over MultilevelLinearOp preconditioned by 2 AMR V-cycles (GSRB 4+4+4), max norm, "
                "rel. residual 1e-10",
    },
    "config1-mixed": {
        "golden": "config1_vc_3lev_128",
        "mixed": True,
        "name": "3-level VC Helmholtz, base 128^3 (as config1); FP32 V-cycles inside FP64 iterative "
                "refinement (residual, reflux, bottom, norms FP64)",
    },
    "config0": {
        "golden": "config0_poisson_64",
        "name": "single-level Poisson (AMRPoissonOp alpha=0 beta=1), 64^3, max box 32, Dirichlet, "
                "GSRB 4+4, BiCGStab bottom, rel. residual 1e-10",
    },
}


def load_cmg():
    import importlib.util
    spec = importlib.util.spec_from_file_location("cmg", os.path.join(ROOT, "chombo_3.2_b200", "cmg.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def golden_meta(name):
    return json.load(open(os.path.join(GOLDEN, name + ".json")))


def covered_cells(boxes, finer_boxes):
    """Valid cells of a level (boxes in layout order, x fastest) under the next finer level (ratio 2)."""
    masks = []
    fine = [(np.array(b[:3]) // 2, np.array(b[3:]) // 2) for b in finer_boxes]
    for b in boxes:
        lo, hi = np.array(b[:3]), np.array(b[3:])
        n = hi - lo + 1
        m = np.zeros((n[2], n[1], n[0]), bool)
        for flo, fhi in fine:
            a, c = np.maximum(lo, flo), np.minimum(hi, fhi)
            if np.all(a <= c):
                m[a[2] - lo[2]:c[2] - lo[2] + 1, a[1] - lo[1]:c[1] - lo[1] + 1, a[0] - lo[0]:c[0] - lo[0] + 1] = True
        masks.append(m.ravel())
    return np.concatenate(masks)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sms = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sms)) if sms else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def write_boxfile(meta):
    f = tempfile.NamedTemporaryFile("w", suffix=".boxes", delete=False)
    f.write(f"{len(meta['boxes'])}\n")
    for bl in meta["boxes"]:
        f.write(f"{len(bl)}\n")
        for b in bl:
            f.write(" ".join(map(str, b)) + "\n")
    f.close()
    return f.name


def oracle_args(meta, boxfile, iters, repeat):
    return [ORACLE, f"n0={meta['n0']}", f"levels={len(meta['boxes'])}", f"maxbox={meta['maxbox']}",
            f"block={meta['block']}", f"op={meta['op']}", f"alpha={meta['alpha']}", f"beta={meta['beta']}",
            f"seed={meta['seed']}", f"pre={meta['pre']}", f"post={meta['post']}", f"bottom={meta['bottom']}",
            f"eps={meta['eps']}", f"hang={meta['hang']}", f"iters={iters}", f"repeat={repeat}", "dumpphi=0",
            f"boxfile={boxfile}", f"out={boxfile}.out"]


def parse_repeats(text):
    reps = []
    for line in text.splitlines():
        if line.startswith("repeat "):
            w = line.split()
            its = [float(x) for x in w[w.index("iterations") + 1:]]
            reps.append({"seconds": float(w[3]), "setup": float(w[5]), "iterations": its})
    return reps


def extrapolate(rep, n_iter):
    """Full-solve time from a capped solve: set-up + first iteration + the
    remaining iterations at the later (steady) iteration time."""
    its = rep["iterations"]
    steady = its[-1] if len(its) > 1 else its[0]
    return rep["setup"] + its[0] + (n_iter - 1) * steady


def cpu_reference(meta, processes, repeats):
    """The reference solve (oracle/_ref, the reference's C++ with the
    restated ChF kernels) on host cores: `processes` concurrent single-thread
    solves of the workload, each capped at 2 V-cycles per repeat and
    extrapolated to the reference's own iteration count."""
    if not os.path.exists(ORACLE):
        return None
    boxfile = write_boxfile(meta)
    n_iter = len(meta["residual_history"]) - 1
    procs = [subprocess.Popen(oracle_args(meta, boxfile, 2, repeats), stdout=subprocess.PIPE,
                              stderr=subprocess.DEVNULL, text=True) for _ in range(processes)]
    outs = [parse_repeats(p.communicate()[0]) for p in procs]
    per_step = []
    for k in range(repeats):
        ts = [extrapolate(o[k], n_iter) for o in outs if len(o) > k]
        per_step.append(len(ts) / max(ts) if ts else float("nan"))
    return {"per_step": per_step, "n_iter": n_iter, "processes": processes,
            "wall_step": [max(o[k]["seconds"] for o in outs if len(o) > k) for k in range(repeats)]}


def cpu_reference_openmp(meta, threads):
    """One reference solve at a time on all host cores: the oracle built with
    the reference's OpenMP box loops (oracle/_ref/omp), OMP_NUM_THREADS =
    threads, capped at 2 V-cycles and extrapolated like cpu_reference.  The
    reference's own OpenMP code is only valid on single-level hierarchies:
    LevelFluxRegister::reflux adds the fine registers through copyTo with an
    AddOp that keeps LDOperator's threadSafe() == true, so the copy's motion
    items run in parallel and items writing the same coarse cells lose
    updates; multi-level solves then stagnate (measured with 8 threads: exit
    status 4 instead of 1).  The timing is reported either way, with that
    outcome stated."""
    if not os.path.exists(OMPORACLE):
        return None
    boxfile = write_boxfile(meta)
    n_iter = len(meta["residual_history"]) - 1
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    args = oracle_args(meta, boxfile, 2, 1)
    args[0] = OMPORACLE
    out = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=env).stdout
    reps = parse_repeats(out)
    if not reps:
        return None
    solve_s = extrapolate(reps[0], n_iter)
    single = len(meta["boxes"]) == 1
    return {"value": 1.0 / solve_s, "unit": "solves/s", "cores": threads, "kind": "reference",
            "sample": f"one reference solve with OMP_NUM_THREADS={threads} (the reference's OpenMP box loops), "
                      f"capped at 2 of {n_iter} V-cycles, extrapolated to the full solve",
            "valid": single,
            "note": "single-level: the reference's OpenMP path converges as the serial one" if single else
                    "multi-level: the reference's OpenMP reflux (LevelFluxRegister AddOp copy in parallel) loses "
                    "flux-register updates and the solve stagnates, so this is the speed of an invalid solve"}


def cpu_reference_bicgstab(meta, wl, processes):
    """The reference's BiCGStab over MultilevelLinearOp (oracle/_ref/cmg_oracle_mlbicgstab) on host cores:
    `processes` concurrent single-thread solves of the workload capped at 1 and at 2 BiCGStab iterations; the
    full solve is extrapolated as t(1) + (n - 1) (t(2) - t(1)) with n the GPU solve's iteration count."""
    if not os.path.exists(MLORACLE):
        return None
    boxfile = write_boxfile(meta)
    b = wl["bicgstab"]
    base = [MLORACLE, f"n0={meta['n0']}", f"levels={len(meta['boxes'])}", f"maxbox={meta['maxbox']}",
            f"block={meta['block']}", f"op={meta['op']}", f"alpha={meta['alpha']}", f"beta={meta['beta']}",
            f"seed={meta['seed']}", f"mgiters={b['mg_iters']}", f"mgsmooth={b['mg_smooth']}", f"eps={b['eps']}",
            f"boxfile={boxfile}"]
    times = {}
    for imax in (1, 2):
        procs = [subprocess.Popen(base + [f"imax={imax}", f"out={boxfile}.{imax}.{k}"], stdout=subprocess.PIPE,
                                  stderr=subprocess.DEVNULL, text=True) for k in range(processes)]
        outs = [p.communicate()[0] for p in procs]
        ts = [float(o.split("seconds=")[1].split()[0]) for o in outs if "seconds=" in o]
        times[imax] = max(ts) if ts else float("nan")
    return times


def run_reference_arm(args, meta, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(ORACLE):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cmg_oracle not built (needs the "
                          "reference sources at build time)"}))
        return
    cores = os.cpu_count() or 1
    # each process holds ~3 GB for this workload; bound the concurrency
    procs = max(1, min(cores, 8))
    if wl.get("solver") == "bicgstab":
        n_iter = wl.get("reference_iterations", 8)
        t = cpu_reference_bicgstab(meta, wl, procs)
        if t is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cmg_oracle_mlbicgstab not built"}))
            return
        solve_s = t[1] + (n_iter - 1) * (t[2] - t[1])
        value = procs / solve_s
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": 1000.0 * solve_s, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["name"], "global_batch": 1, "parallelism": f"{procs} concurrent host processes"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": "reference",
                             "sample": f"{procs} concurrent single-thread reference BiCGStab solves capped at 1 and 2 "
                                       f"iterations, extrapolated to {n_iter} iterations"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    res = cpu_reference(meta, procs, args.warmup + args.steps)
    timed = res["per_step"][args.warmup:]
    value = float(np.mean(timed))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(res["wall_step"][args.warmup:])),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["name"], "global_batch": 1, "parallelism": f"{procs} concurrent host processes"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": "reference",
                         "sample": f"each step: {procs} concurrent single-thread reference solves capped at 2 of "
                                   f"{res['n_iter']} V-cycles, extrapolated to the full solve"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def replica_rate(local_ms, units_per_rank, dist=None, device="cuda"):
    """Whole-job rate of N independent replicas: each rank's device time for its own units, the slowest rank
    (MAX all-reduce) taken as the job's time, all ranks' units counted.  Returns (units/s, max ms)."""
    import torch
    world = dist.get_world_size() if dist else 1
    ms = float(local_ms)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return world * units_per_rank / (ms / 1000.0), ms


def round16(x):
    return int(max(32, 16 * round(x / 16.0)))


def batch_specs(n, seed):
    """512 independent 2-level problems: base n0 log-uniform in [32, 128]
    rounded to a multiple of 16, max box from {16, 24, 32}, Poisson
    (AMRPoissonOp alpha=0 beta=1) or variable-coefficient Helmholtz
    (VCAMRPoissonOp2 alpha=1 beta=-1, coefficients in [0.1, 10]) with p=1/2,
    each with its own seed."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        n0 = min(128, round16(math.exp(rng.uniform(math.log(32), math.log(128)))))
        vc = bool(rng.random() < 0.5)
        specs.append(dict(n0=n0, levels=2, max_box=int(rng.choice([16, 24, 32])), block_factor=8, fill_ratio=0.75,
                          thresh=0.1, seed=1000 + i, op=1 if vc else 0, alpha=1.0 if vc else 0.0,
                          beta=-1.0 if vc else 1.0))
    return specs


def cpu_reference_sample(cmg, specs, processes):
    """The reference solve (oracle/_ref/cmg_oracle, full solves to 1e-10) of a sample of independent problems on
    the host cores, `processes` at a time, each from the product's grid generation (box lists identical to the
    reference's BRMeshRefine).  Returns (solves/s over the wall time, wall seconds)."""
    if not os.path.exists(ORACLE):
        return None
    jobs = []
    for sp in specs:
        boxes = cmg.synthetic_hierarchy(sp["n0"], sp["levels"], sp["max_box"], sp["block_factor"],
                                        sp["fill_ratio"], sp["seed"], sp["thresh"])
        bf = write_boxfile({"boxes": boxes})
        jobs.append([ORACLE, f"n0={sp['n0']}", f"levels={len(boxes)}", f"maxbox={sp['max_box']}",
                     f"block={sp['block_factor']}", f"op={sp['op']}", f"alpha={sp['alpha']}", f"beta={sp['beta']}",
                     f"seed={sp['seed']}", f"eps={sp.get('eps', 1e-10)}", "dumpphi=0", f"boxfile={bf}",
                     f"out={bf}.out"])
    t0 = time.perf_counter()
    running = []
    for cmd in jobs:
        running.append(subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
        if len(running) >= processes:
            running.pop(0).wait()
    for p in running:
        p.wait()
    wall = time.perf_counter() - t0
    return len(jobs) / wall, wall


def serving_stream(rate, n, seed):
    """Open-loop request stream: exponential inter-arrival times at `rate`, levels U{1,2,3}, base n0
    log-uniform in [32, 256] (x16), Poisson or VC Helmholtz and tolerance 1e-8 or 1e-10 with p = 1/2 each."""
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        n0 = min(256, round16(math.exp(rng.uniform(math.log(32), math.log(256)))))
        vc = bool(rng.random() < 0.5)
        eps = 1e-8 if rng.random() < 0.5 else 1e-10
        reqs.append(dict(arrival=t, n0=n0, levels=int(rng.integers(1, 4)), max_box=32, block_factor=8,
                         fill_ratio=0.75, thresh=0.1, seed=5000 + i, op=1 if vc else 0, alpha=1.0 if vc else 0.0,
                         beta=-1.0 if vc else 1.0, eps=eps))
    return reqs


def run_reference_batch(args):
    """Reference arm of the batch (config3) and serving (config4) workloads: the reference solve of a seeded
    sample of their problems on the host cores (all cores for the batch, one at a time for serving, whose
    reference baseline is sequential solves)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if not os.path.exists(ORACLE):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cmg_oracle not built"}))
        return
    cmg = load_cmg()
    if args.workload == "config3":
        specs = batch_specs(args.batch, 20261203)[::16]
        procs = max(1, min(os.cpu_count() or 1, 8))
        name = f"{args.batch} independent 2-level hierarchies (sample of {len(specs)})"
    else:
        # the first requests of the lowest-rate stream, sized so the sample ends within minutes
        specs = [q for q in serving_stream(50.0, args.requests, 50) if q["n0"] * q["levels"] <= 256][:6]
        procs = 1
        name = (f"open-loop serving requests (the first {len(specs)} of the 50 req/s stream with n0 x levels <= 256, "
                "solved one at a time)")
    rate, wall = cpu_reference_sample(cmg, specs, procs)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "solves/s", "n_gpus": args.gpus, "steps": 1,
        "warmup": 0, "ms_per_step": 1000.0 * wall, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": name, "global_batch": len(specs), "parallelism": f"{procs} host processes"},
        "cpu_baseline": {"value": rate, "unit": "solves/s", "cores": procs, "kind": "reference",
                         "sample": f"{len(specs)} problems, full reference solves to 1e-10"},
        "e2e": {"value": rate, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_batch(args):
    """Batching: N independent hierarchies resident on the GPU, solved
    concurrently (one stream each, every iteration a CUDA-graph replay,
    FP32 V-cycles inside FP64 refinement), against the plain FP64 drop-in
    solving the same hierarchies one at a time."""
    import concurrent.futures as cf
    import torch
    torch.cuda.set_device(0)
    cmg = load_cmg()
    specs = batch_specs(args.batch, 20261203)
    params = cmg.solve_params(eps=1e-10)
    wave = args.wave
    t_batch = t_seq = 0.0
    cells = 0
    iters_mixed, iters_fp64, not_converged = [], [], 0
    pool = cf.ThreadPoolExecutor(max_workers=args.inflight)

    def build(sp):
        boxes = cmg.synthetic_hierarchy(sp["n0"], sp["levels"], sp["max_box"], sp["block_factor"],
                                        sp["fill_ratio"], sp["seed"], sp["thresh"])
        h = cmg.Hierarchy(sp["n0"], boxes, op=sp["op"], alpha=sp["alpha"], beta=sp["beta"])
        h.fill_synthetic(sp["seed"], device=not args.host_fill)
        return h

    if args.forest:
        return run_batch_forest(args, cmg, specs, params, pool)
    for w0 in range(0, len(specs), wave):
        hs = list(pool.map(build, specs[w0:w0 + wave]))
        cells += sum(sum(h.num_cells(l) for l in range(h.nlev)) for h in hs)
        for h in hs:
            h.use_graphs(True)
            h.set_relax_mode(args.relax_mode)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs = list(pool.map(lambda h: h.solve(params, mixed=True), hs))
        torch.cuda.synchronize()
        t_batch += time.perf_counter() - t0
        iters_mixed += [o["iterations"] for o in outs]
        not_converged += sum(1 for o in outs if not (o["exit_status"] & 1))
        for h in hs:
            h.use_graphs(False)
        t0 = time.perf_counter()
        for h in hs:
            o = h.solve(params)
            iters_fp64.append(o["iterations"])
        torch.cuda.synchronize()
        t_seq += time.perf_counter() - t0
        for h in hs:
            h.close()
    value = len(specs) / t_batch
    base = len(specs) / t_seq
    cpu = None
    if not args.no_cpu_baseline:
        procs = max(1, min(os.cpu_count() or 1, 8))
        sample = specs[::16]
        r = cpu_reference_sample(cmg, sample, procs)
        if r:
            cpu = {"value": r[0], "unit": "solves/s", "cores": procs, "kind": "reference",
                   "sample": f"{len(sample)} of the {len(specs)} problems (every 16th), full reference solves to "
                             f"1e-10, {procs} at a time on the host cores; rate = problems / wall time "
                             f"({r[1]:.1f} s)"}
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": 1000.0 * t_batch, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"{len(specs)} independent 2-level hierarchies, base 32^3-128^3 log-uniform (x16), "
                               "max box 16/24/32, Poisson or VC Helmholtz, rel. residual 1e-10",
                   "resident_per_wave": wave, "concurrent_streams": args.inflight, "cells": cells,
                   "relax_mode": args.relax_mode,
                   "timing": "wall clock around the concurrent solves of each resident wave (host "
                             "set-up of the hierarchies not timed)"},
        "cpu_baseline": cpu,
        "plain_fp64_one_at_a_time": {"value": base, "unit": "solves/s", "ratio": value / base},
        "vcycles_mixed_mean": float(np.mean(iters_mixed)), "vcycles_fp64_mean": float(np.mean(iters_fp64)),
        "not_converged": not_converged,
    }
    print(json.dumps(line), flush=True)


def run_batch_forest(args, cmg, specs, params, pool):
    """Batching with forests: the problems grouped by (base size, max box, operator), each group one forest
    (cmg_forest_create: its hierarchies' levels merged, one kernel launch per V-cycle operation for the whole
    group, a bottom-solve block per hierarchy, per-hierarchy stopping), the forests solved concurrently on
    their own streams, FP32 V-cycles inside FP64 refinement.  Every hierarchy's result is the one its own
    solve gives (tests/test_forest_gpu.py)."""
    import torch
    groups = {}
    for sp in specs:
        groups.setdefault((sp["n0"], sp["max_box"], sp["op"]), []).append(sp)
    cap = max(1, args.forest_size)
    parts = []
    for key in sorted(groups):
        g = groups[key]
        for a in range(0, len(g), cap):
            parts.append(g[a:a + cap])

    def build(part):
        sp0 = part[0]
        hb = [cmg.synthetic_hierarchy(sp["n0"], sp["levels"], sp["max_box"], sp["block_factor"], sp["fill_ratio"],
                                      sp["seed"], sp["thresh"]) for sp in part]
        f = cmg.Forest(sp0["n0"], hb, op=sp0["op"], alpha=sp0["alpha"], beta=sp0["beta"])
        f.fill_synthetic([sp["seed"] for sp in part])
        f.use_graphs(True)
        f.set_relax_mode(args.relax_mode)
        return f

    t_build = time.perf_counter()
    forests = list(pool.map(build, parts))
    t_build = time.perf_counter() - t_build
    cells = sum(sum(f.num_cells(l) for l in range(f.nlev)) for f in forests)
    # first solve of each forest: autotuning and graph capture, not timed
    list(pool.map(lambda f: f.solve(params, mixed=True), forests))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    outs = list(pool.map(lambda f: f.solve(params, mixed=True), forests))
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    res = [o for out in outs for o in out]
    iters = [o["iterations"] for o in res]
    not_converged = sum(1 for o in res if not (o["exit_status"] & 1))
    for f in forests:
        f.close()
    value = len(specs) / t_batch
    cpu = None
    if not args.no_cpu_baseline:
        procs = max(1, min(os.cpu_count() or 1, 8))
        sample = specs[::16]
        r = cpu_reference_sample(cmg, sample, procs)
        if r:
            cpu = {"value": r[0], "unit": "solves/s", "cores": procs, "kind": "reference",
                   "sample": f"{len(sample)} of the {len(specs)} problems (every 16th), full reference solves to "
                             f"1e-10, {procs} at a time on the host cores; rate = problems / wall time "
                             f"({r[1]:.1f} s)"}
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": 1000.0 * t_batch, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"{len(specs)} independent 2-level hierarchies, base 32^3-128^3 log-uniform (x16), "
                               "max box 16/24/32, Poisson or VC Helmholtz, rel. residual 1e-10",
                   "batching": f"{len(forests)} forests (hierarchies grouped by base size, max box and operator, "
                               f"at most {cap} per forest), solved concurrently on {args.inflight} host threads, "
                               "one stream per forest",
                   "cells": cells, "relax_mode": args.relax_mode,
                   "timing": "wall clock around one solve of every forest (all resident; host set-up, autotuning "
                             "and graph capture in an untimed first solve)"},
        "cpu_baseline": cpu,
        "vcycles_mixed_mean": float(np.mean(iters)), "not_converged": not_converged,
        "host_setup_s": t_build,
    }
    if getattr(args, "quiet_line", False):
        return line
    print(json.dumps(line), flush=True)


def extra_workloads(args, cmg):
    """The precision and batching workloads measured in the default run, so that their numbers come from the
    same run as the headline: config 2 (3-level 256^3 VC Helmholtz, 149M cells, FP32 V-cycles in FP64
    refinement, 3 timed solves after one warm-up, CUDA events on the solver's stream) and config 3 (512
    independent 2-level hierarchies in forests, wall clock around one solve of every forest)."""
    import concurrent.futures as cf
    import torch
    out = {}
    try:
        meta = golden_meta(WORKLOADS["config2"]["golden"])
        h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
        h.fill_synthetic(meta["seed"])
        p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                             eps=meta["eps"], hang=meta["hang"])
        h.use_graphs(True)
        o = h.solve(p, mixed=True)
        stream = torch.cuda.ExternalStream(h.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        n = 3
        for _ in range(n):
            o = h.solve(p, mixed=True)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b) / n
        out["config2"] = {"workload": WORKLOADS["config2"]["name"], "value": 1000.0 / ms, "unit": "solves/s",
                          "ms_per_solve": ms, "fp64_refinement_steps": o["iterations"],
                          "exit_status": o["exit_status"], "reference_vcycles": len(meta["residual_history"]) - 1,
                          "cells": sum(h.num_cells(l) for l in range(len(meta["boxes"]))), "dtype": "f32+f64",
                          "timing": "CUDA events on the solver's stream around 3 solves after one untimed solve"}
        h.close()
    except Exception as e:  # reported, not fatal: the headline line stands on its own
        out["config2"] = {"error": str(e)[:300]}
    try:
        specs = batch_specs(512, 20261203)
        pool = cf.ThreadPoolExecutor(max_workers=16)
        a2 = argparse.Namespace(**vars(args))
        a2.forest_size, a2.inflight, a2.relax_mode, a2.no_cpu_baseline, a2.quiet_line = 64, 16, 0, True, True
        line = run_batch_forest(a2, cmg, specs, cmg.solve_params(eps=1e-10), pool)
        out["config3"] = {k: line[k] for k in ("value", "unit", "ms_per_step", "vcycles_mixed_mean", "not_converged",
                                               "host_setup_s", "dtype")}
        out["config3"]["workload"] = line["config"]["workload"]
        out["config3"]["batching"] = line["config"]["batching"]
        out["config3"]["timing"] = line["config"]["timing"]
    except Exception as e:
        out["config3"] = {"error": str(e)[:300]}
    try:
        out["helmholtz_512_periodic"] = published_vcycle(cmg)
    except Exception as e:
        out["helmholtz_512_periodic"] = {"error": str(e)[:300]}
    return out


def published_vcycle(cmg, n0=512, steps=1, warmup=1, relax_mode=0, graphs=True):
    """The configuration of the reference's one published AMRPoisson timing: a single level 512^3 on the unit
    domain, periodic in every direction, domainSplit into 32^3 boxes (block factor 8), alpha = 1, beta = -0.1,
    4 smoothings per relaxation (releasedExamples/Proto/Poisson/doc/proto_poisson.tex:18-55 and
    exec/periodic.inputs), 1.223 s per V-cycle on a 32-core Haswell node (n0 other than 512: the same recipe at
    that size).  Seeded synthetic right-hand side; warmup untimed solves, then `steps` timed solves in CUDA events
    on the solver's stream, divided by their V-cycle count (each V-cycle is followed by the residual and its max
    norm, as in the example's loop)."""
    import torch
    boxes = cmg.domain_split((0, 0, 0), (n0 - 1,) * 3, 32, 8)
    h = cmg.Hierarchy(n0, [boxes], op=0, alpha=1.0, beta=-0.1, bc="PPPPPP")
    try:
        h.fill_synthetic(20261203)
        p = cmg.solve_params(pre=4, post=4, bottom=4, iter_max=100, eps=1e-10, hang=1e-10)
        h.set_relax_mode(relax_mode)
        h.use_graphs(graphs)
        for _ in range(max(warmup, 1)):
            h.solve(p)
        stream = torch.cuda.ExternalStream(h.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(steps):
            o = h.solve(p)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b) / steps
        nv = max(o["iterations"], 1)
        vb = h.vcycle_bytes(p)
        peak = measured_peaks()[0]
        return {"workload": f"single level {n0}^3 periodic Helmholtz (alpha 1, beta -0.1), {len(boxes)} boxes of "
                            "32^3, 4 smoothings", "ms_per_vcycle": ms / nv, "vcycles": o["iterations"],
                "exit_status": o["exit_status"], "ms_per_solve": ms, "cells": h.num_cells(0),
                "vcycle_gbs": vb / (ms / nv) / 1e6, "vcycle_frac": vb / (ms / nv) / 1e6 / peak,
                "published_s_per_vcycle": 1.223 if n0 == 512 else None,
                "published_hardware": "1 Cori Haswell node, 32 MPI ranks", "dtype": "f64",
                "timing": f"CUDA events on the solver's stream around {steps} solve(s) after {max(warmup, 1)} "
                          "untimed"}
    finally:
        h.close()


def periodic_reference(cmg, n0, n_iter, threads):
    """The reference on the periodic configuration: the oracle built with the reference's OpenMP box loops (valid
    on one level), OMP_NUM_THREADS = threads, capped at 2 V-cycles; returns seconds per (steady) V-cycle, the
    set-up, and the full solve extrapolated to n_iter V-cycles."""
    if not os.path.exists(OMPORACLE):
        return None
    boxes = cmg.domain_split((0, 0, 0), (n0 - 1,) * 3, 32, 8)
    meta = {"n0": n0, "boxes": [[list(b) for b in boxes]], "maxbox": 32, "block": 8, "op": 0, "alpha": 1.0,
            "beta": -0.1, "seed": 20261203, "pre": 4, "post": 4, "bottom": 4, "eps": 1e-10, "hang": 1e-10}
    boxfile = write_boxfile(meta)
    a = oracle_args(meta, boxfile, 2, 1) + ["bc=PPPPPP"]
    a[0] = OMPORACLE
    out = subprocess.run(a, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
                         env=dict(os.environ, OMP_NUM_THREADS=str(threads))).stdout
    reps = parse_repeats(out)
    if not reps:
        return None
    its = reps[0]["iterations"]
    return {"s_per_vcycle": its[-1], "setup_s": reps[0]["setup"], "solve_s": extrapolate(reps[0], n_iter),
            "cores": threads}


def run_periodic(args):
    """--workload periodic: the published configuration (published_vcycle) as its own line."""
    cmg = load_cmg()
    r = published_vcycle(cmg, n0=args.n0, steps=args.steps, warmup=args.warmup, relax_mode=args.relax_mode,
                         graphs=not args.no_graphs)
    line = {"metric": METRIC, "value": 1000.0 / r["ms_per_solve"], "unit": "solves/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_solve"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": r["workload"]}, "gpu_launches": cmg.launch_count()}
    line.update({k: r[k] for k in ("ms_per_vcycle", "vcycles", "exit_status", "cells", "vcycle_gbs", "vcycle_frac",
                                   "published_s_per_vcycle", "published_hardware", "timing")})
    if not args.no_cpu_baseline:
        ref = periodic_reference(cmg, args.n0, r["vcycles"], os.cpu_count() or 1)
        if ref:
            line["cpu_baseline"] = {"value": 1.0 / ref["solve_s"], "unit": "solves/s", "cores": ref["cores"],
                                    "kind": "reference", "s_per_vcycle": ref["s_per_vcycle"],
                                    "sample": f"one reference solve with OMP_NUM_THREADS={ref['cores']} (single "
                                              "level: the reference's OpenMP box loops are valid), capped at 2 "
                                              f"V-cycles, extrapolated to the solve's {r['vcycles']}"}
    print(json.dumps(line))


def run_periodic_reference(args):
    """--impl reference of --workload periodic: periodic_reference on all host cores, as its own line."""
    cmg = load_cmg()
    n_iter = 6  # V-cycles of this solve to 1e-10 (the GPU solve reproduces the reference's history bit for bit)
    ref = periodic_reference(cmg, args.n0, n_iter, os.cpu_count() or 1)
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/omp/cmg_oracle is not built"}))
        return
    v = 1.0 / ref["solve_s"]
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": 1,
                      "steps": 1, "warmup": 0, "ms_per_step": 1000.0 * ref["solve_s"], "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": f"single level {args.n0}^3 periodic Helmholtz (alpha 1, beta -0.1), "
                                             "boxes of 32^3, 4 smoothings"},
                      "s_per_vcycle": ref["s_per_vcycle"], "setup_s": ref["setup_s"],
                      "cpu_baseline": {"value": v, "unit": "solves/s", "cores": ref["cores"], "kind": "reference",
                                       "sample": "one solve capped at 2 V-cycles, extrapolated to 6"},
                      "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def fineinterp_reference(meta, repeat):
    """The reference's FineInterp (oracle/_ref/cmg_oracle_fineinterp, interpToFine with PCInterp limiting) on
    one host core, for every level above 0 of the hierarchy: `repeat` timed interpolations per level; returns
    (fine cells per second, seconds per step)."""
    if not os.path.exists(FIORACLE):
        return None
    boxfile = write_boxfile(meta)
    secs, cells = 0.0, 0
    for lev in range(1, len(meta["boxes"])):
        out = subprocess.run([FIORACLE, f"n0={meta['n0']}", f"levels={len(meta['boxes'])}",
                              f"maxbox={meta['maxbox']}", f"block={meta['block']}", f"seed={meta['seed']}",
                              f"level={lev}", f"repeat={repeat}", f"boxfile={boxfile}", f"out={boxfile}.fi"],
                             capture_output=True, text=True, check=True).stdout
        w = out.split("fine cells=")[1].split()
        cells += int(w[0])
        secs += float(w[1].split("=")[1])
    return cells / secs, secs


def run_fineinterp(args):
    """FineInterp::interpToFine of every level above 0 of the config-1
    hierarchy (what a regrid does to initialise new levels): device-resident
    fine cells per second from CUDA events around each level's two kernels,
    L2 flushed between steps; end to end through the standalone
    cmg_fine_interp object with the coarse data sent from and the fine data
    read back to host memory every step."""
    meta = golden_meta("config1_vc_3lev_128")
    nlev = len(meta["boxes"])
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        r = fineinterp_reference(meta, max(1, args.steps))
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cmg_oracle_fineinterp not built"}))
            return
        cpu = {"value": r[0], "unit": "cells/s", "cores": 1, "kind": "reference",
               "sample": f"full workload, {max(1, args.steps)} interpolations per level (the reference's "
                         "interpToFine loops over boxes on one thread)"}
        print(json.dumps({"impl": "reference", "metric": "FineInterp fine cells/s", "value": r[0], "unit": "cells/s",
                          "n_gpus": 1, "steps": args.steps, "warmup": 0, "ms_per_step": 1000.0 * r[1],
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": {"workload": "fineinterp-config1"}, "cpu_baseline": cpu,
                          "e2e": {"value": r[0], "unit": "cells/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    torch.cuda.set_device(0)
    cmg = load_cmg()
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
    h.fill_synthetic(meta["seed"])
    rhs = [h.get_rhs(l) for l in range(nlev)]
    for l in range(nlev - 1):
        h.set_phi(l, rhs[l])
    fine_cells = sum(h.num_cells(l) for l in range(1, nlev))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step():
        for l in range(1, nlev):
            h.interp_to_fine(l)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    launches0 = cmg.launch_count()
    h.profile_enable(True)
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        step()
    n_runs, ms, nbytes = h.profile_read(5)
    h.profile_enable(False)
    launches = cmg.launch_count() - launches0
    clocks = sampler.stop()
    value = fine_cells * args.steps / (ms / 1e3)

    # the reference's output at level 2 from the level-1 right-hand side
    ref = np.load(os.path.join(ROOT, "tests", "golden", "fineinterp_config1_vc_3lev_128_l2.npz"))["fine"]
    h.set_phi(1, rhs[1])
    h.interp_to_fine(2)
    parity = bool(np.array_equal(h.phi(2)[::997], ref))
    h.close()

    # end to end: standalone objects, pinned host data in and out every step
    nf = meta["n0"]
    fis, coarse, outs = [], [], []
    for l in range(1, nlev):
        nf *= 2
        fis.append(cmg.FineInterp((0, 0, 0, nf - 1, nf - 1, nf - 1), meta["boxes"][l], meta["boxes"][l - 1]))
        c = torch.empty(rhs[l - 1].size, dtype=torch.float64, pin_memory=True).numpy()
        c[:] = rhs[l - 1]
        coarse.append(c)
        outs.append(torch.empty(fis[-1].nfine, dtype=torch.float64, pin_memory=True).numpy())
    for fi, c, o in zip(fis, coarse, outs):
        fi.interp_to_fine(c, out=o)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for fi, c, o in zip(fis, coarse, outs):
            fi.interp_to_fine(c, out=o)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    for fi in fis:
        fi.close()
    h2d = sum(c.size for c in coarse) * 8
    d2h = fine_cells * 8
    e2e = {"value": fine_cells * args.steps / e2e_s, "unit": "cells/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "timing": "wall clock, pinned host arrays in and out"}

    peak, peak_kind = measured_peaks()
    achieved = (nbytes / 1e9) / (ms / 1e3)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        t = json.load(open(tpath)).get("fineinterp")
        traffic = t["dram_bytes_per_step"] if t else None
    cpu = None
    if not args.no_cpu_baseline:
        r = fineinterp_reference(meta, 1)
        if r:
            cpu = {"value": r[0], "unit": "cells/s", "cores": 1, "kind": "reference",
                   "sample": "full workload, one interpolation per level"}
    line = {"metric": "FineInterp fine cells/s", "value": value, "unit": "cells/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "fineinterp-config1: interpToFine of levels 1 and 2 of the 3-level 128^3 "
                                   "hierarchy from the seeded right-hand side", "fine_cells_per_step": fine_cells,
                       "l2": "flushed (256 MB write) before every step",
                       "timing": "sum of CUDA-event device times around each level's interpolation launches"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_unit": "DRAM bytes per step (both levels)",
                         "peak_kind": peak_kind,
                         "kernel": "k_fi_fused: one launch per level, the coarse staging block of a fine box in "
                                   "shared memory (algorithmic bytes: 8 B written per fine cell + 8 B read per "
                                   "coarse parent)",
                         "timed_regions": int(n_runs), "algorithmic_bytes_per_step": nbytes / args.steps},
            "parity_level2_vs_reference": parity, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches}
    print(json.dumps(line), flush=True)


def run_serving(args):
    """Serving: open-loop Poisson arrivals at each rate; each request a 1-3
    level hierarchy, base 32^3-256^3 log-uniform (x16), seeded inputs,
    tolerance 1e-8 or 1e-10, admitted against a 120 GB device-memory budget
    (cmg_serve); reports p50/p99 latency (arrival to solution on the host) and
    completed solves/s per rate, beside the plain FP64 solve one request at a
    time."""
    import torch
    torch.cuda.set_device(0)
    cmg = load_cmg()
    rates = [float(r) for r in args.rates.split(",")]

    def stream(rate, n, seed):
        reqs = serving_stream(rate, n, seed)
        for q in reqs:
            q.update(params=cmg.solve_params(eps=q["eps"]), mixed=True, graphs=True, device_tags=not args.host_tags)
        return reqs

    def stats(res, wall):
        lat = np.array([r["finished"] - q for r, q in res])
        ok = sum(1 for r, _ in res if r["error"] == 0 and r["exit_status"] & 1)
        return {"p50_ms": 1000.0 * float(np.percentile(lat, 50)), "p99_ms": 1000.0 * float(np.percentile(lat, 99)),
                "solves_per_s": len(res) / wall, "converged": ok, "requests": len(res),
                "mean_setup_ms": 1000.0 * float(np.mean([r["setup_seconds"] for r, _ in res])),
                "mean_solve_ms": 1000.0 * float(np.mean([r["solve_seconds"] for r, _ in res])),
                "mean_grid_ms": 1000.0 * float(np.mean([r["grid_seconds"] for r, _ in res])),
                "mean_build_ms": 1000.0 * float(np.mean([r["build_seconds"] for r, _ in res])),
                "batched_requests": sum(1 for r, _ in res if r["batch_size"] > 1)}

    per_rate = {}
    for rate in rates:
        reqs = stream(rate, args.requests, int(rate))
        res, wall = cmg.serve(reqs, hbm_budget=120e9, max_inflight=args.inflight, open_loop=True,
                              batch_window=args.batch_window, max_batch=16)
        per_rate[str(int(rate))] = stats(list(zip(res, [q["arrival"] for q in reqs])), wall)
    # The plain FP64 GPU solve, one request at a time, on the first rate's stream.
    reqs = stream(rates[0], args.requests, int(rates[0]))
    for q in reqs:
        q["mixed"], q["graphs"] = False, False
    res, wall = cmg.serve(reqs, hbm_budget=120e9, max_inflight=1, open_loop=True)
    base = stats(list(zip(res, [q["arrival"] for q in reqs])), wall)
    top = per_rate[str(int(rates[-1]))]
    line = {
        "metric": METRIC, "value": top["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": 1,
        "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "open-loop Poisson arrivals, 1-3 level hierarchies, base 32^3-256^3 log-uniform "
                               "(x16), Poisson or VC Helmholtz, tolerance 1e-8 or 1e-10, 120 GB budget",
                   "requests_per_rate": args.requests, "workers": args.inflight,
                   "latency": "arrival to phi on the host, including grid generation and set-up",
                   "tagging": "host" if args.host_tags else "device",
                   "batch_window_s": args.batch_window},
        "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"], "per_rate": per_rate,
        "plain_fp64_one_at_a_time": base,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config1",
                    choices=sorted(WORKLOADS) + ["config3", "config4", "fineinterp", "periodic"])
    ap.add_argument("--n0", type=int, default=512, help="periodic: base size (512: the published configuration)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graphs", action="store_true", help="launch every kernel instead of replaying graphs")
    ap.add_argument("--relax-mode", type=int, default=0, choices=[0, 1, 2, 3],
                    help="relaxation variant: 0 autotuned per level, 1 ghost fills, 2 in-pass ghosts")
    ap.add_argument("--batch", type=int, default=512, help="config3: number of hierarchies")
    ap.add_argument("--host-fill", action="store_true", help="config3: generate the inputs on the host")
    ap.add_argument("--wave", type=int, default=128, help="config3: hierarchies resident at once")
    ap.add_argument("--forest", type=int, default=1, help="config3: 1 = batch the problems in forests")
    ap.add_argument("--batch-window", type=float, default=0.0,
                    help="config4: seconds a request waits for others of its class to be solved with it")
    ap.add_argument("--extras", type=int, default=1,
                    help="config1, one GPU: also measure config 2 (mixed) and config 3 (forests) in the same run")
    ap.add_argument("--forest-size", type=int, default=64, help="config3: most hierarchies in one forest")
    ap.add_argument("--inflight", type=int, default=16, help="config3/4: concurrent solves")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="config4: arrival rates (req/s)")
    ap.add_argument("--host-tags", action="store_true", help="config4: tag for grid generation on the host")
    ap.add_argument("--requests", type=int, default=48, help="config4: requests per rate")
    args = ap.parse_args()
    if args.workload == "fineinterp":
        return run_fineinterp(args)
    if args.workload == "periodic":
        return run_periodic_reference(args) if args.impl == "reference" else run_periodic(args)
    if args.workload in ("config3", "config4"):
        if args.impl == "reference":
            return run_reference_batch(args)
        return run_batch(args) if args.workload == "config3" else run_serving(args)
    wl = WORKLOADS[args.workload]
    meta = golden_meta(wl["golden"])
    if args.impl == "reference":
        return run_reference_arm(args, meta, wl)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    args.warmup = max(args.warmup, 3)

    cmg = load_cmg()
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
    h.fill_synthetic(meta["seed"])
    params = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                              eps=meta["eps"], hang=meta["hang"])
    mixed = bool(wl.get("mixed", False))
    bicg = wl.get("solver") == "bicgstab"
    mlp = cmg.mlsolve_params(**wl["bicgstab"]) if bicg else None

    def solve_once():
        return h.solve_bicgstab(mlp) if bicg else h.solve(params, mixed=mixed)

    h.use_graphs(not args.no_graphs)
    h.set_relax_mode(args.relax_mode)
    stream = torch.cuda.ExternalStream(h.stream())
    ncells = [h.num_cells(l) for l in range(len(meta["boxes"]))]

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    for _ in range(args.warmup):
        out = solve_once()
    assert out["exit_status"] == meta["exit_status"], out
    n_iter = out["iterations"]

    # Device-resident timed region.  Working set (~2.5 GB of FP64 fields)
    # exceeds L2, so no flush is needed between steps.
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    launches0 = cmg.launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(args.steps):
            solve_once()
            ev[k + 1].record(stream)
    barrier()
    launches = cmg.launch_count() - launches0
    clocks = sampler.stop()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])

    # Per-class breakdown from separate solves with CUDA events around every
    # kernel class (events add a little time, so these solves are not the
    # timed ones above).
    n_prof = min(args.steps, 3)
    h.profile_enable(True)
    pe = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    pe[0].record(stream)
    for _ in range(n_prof):
        solve_once()
    pe[1].record(stream)
    barrier()
    prof_ms = pe[0].elapsed_time(pe[1])
    classes = {name: h.profile_read(i) for i, name in enumerate(PROFILE_CLASSES)}
    h.profile_enable(False)
    value, total_ms = replica_rate(total_ms, args.steps, dist)

    # End to end through the C ABI: every step uploads the right-hand side
    # of every level from pinned host memory, solves, and reads phi back into
    # pinned host memory.
    host_rhs = [torch.empty(n, dtype=torch.float64, pin_memory=True) for n in ncells]
    host_phi = [torch.empty(n, dtype=torch.float64, pin_memory=True) for n in ncells]
    for l in range(len(ncells)):
        h.get_rhs_ptr(l, host_rhs[l].data_ptr(), 0)
    h2d = sum(ncells) * 8
    d2h = sum(ncells) * 8
    barrier()
    e2e_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e2e_ev[0].record(stream)
    for k in range(args.steps):
        for l in range(len(ncells)):
            h.set_rhs_ptr(l, host_rhs[l].data_ptr(), 0)
        out = solve_once()
        for l in range(len(ncells)):
            h.get_phi_ptr(l, host_phi[l].data_ptr(), 0)
    e2e_ev[1].record(stream)
    barrier()
    e2e_rate, e2e_ms = replica_rate(e2e_ev[0].elapsed_time(e2e_ev[1]), args.steps, dist)
    assert out["exit_status"] == meta["exit_status"], out
    e2e = {"value": e2e_rate, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    peak, peak_kind = measured_peaks()
    n_fine, ms_fine, bytes_fine = classes["relax_finest"]
    achieved = (bytes_fine / 1e9) / (ms_fine / 1e3) if ms_fine > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        t = json.load(open(tpath)).get(args.workload)
        traffic = t["dram_bytes_per_launch"] if t else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": f"k_gsrb_pair<{'float' if mixed else 'double'},{meta['op']}>: one red-black colour pass "
                          "over the finest AMR level (two launches per sweep; the one-colour ghost fill between them "
                          "is timed separately)",
                "peak_kind": peak_kind, "launches": int(n_fine),
                "avg_launch_us": 1000.0 * ms_fine / max(n_fine, 1),
                "algorithmic_bytes_per_launch": bytes_fine / max(n_fine, 1)}
    breakdown = {}
    for name, v in classes.items():
        gbs = (v[2] / 1e9) / (v[1] / 1e3) if v[1] > 0 and v[2] > 0 else None
        breakdown[name] = {"launches": int(v[0]) // n_prof, "ms_per_solve": v[1] / n_prof,
                           "share": v[1] / prof_ms if prof_ms > 0 else 0.0, "gbs": gbs,
                           "frac": gbs / peak if gbs else None}
    # The whole V-cycle: algorithmic bytes of one V-cycle (cmg_vcycle_bytes:
    # every relaxation colour pass, residual and operator pass of every level
    # and multigrid depth, each array read once and each output written once)
    # over the solve time per V-cycle (the solve's initial residual and norm
    # reads included, so this is a lower bound on the V-cycle's own rate).
    vbytes = None if bicg else h.vcycle_bytes(params)
    vcycle = None
    if vbytes:
        vms = (total_ms / args.steps) / max(n_iter, 1)
        vgbs = (vbytes / 1e9) / (vms / 1e3)
        relaxed = sum(ncells[:-1]) * (params.pre + params.post) + ncells[-1] * (params.pre + params.post)
        vcycle = {"algorithmic_bytes": vbytes, "ms": vms, "gbs": vgbs, "frac": vgbs / peak, "peak_kind": peak_kind,
                  "cell_updates_per_s": relaxed / (vms / 1e3),
                  "note": "solve time per V-cycle (initial residual and norm read-backs included)"}
    accuracy = None
    if mixed:
        # L-infinity deviation of the mixed-precision phi from the FP64
        # reference solve's phi (golden samples), relative to max|phi| per
        # level: over the composite solution (cells not covered by a finer
        # level) and over the covered coarse cells, which the composite
        # residual does not constrain.
        gold = np.load(os.path.join(GOLDEN, wl["golden"] + ".npz"))
        nlev, stride = len(meta["boxes"]), meta["sample_stride"]
        comp, covd = 0.0, 0.0
        for lev in range(nlev):
            phi = h.phi(lev)
            cov = covered_cells(meta["boxes"][lev], meta["boxes"][lev + 1]) if lev + 1 < nlev else \
                np.zeros(phi.size, bool)
            full = meta["full"]
            ref = gold[f"phi{lev}"] if full else gold[f"phi{lev}_sample"]
            if not full:
                phi, cov = phi[::stride], cov[::stride]
            dev = np.abs(phi - ref) / meta["phi_absmax"][lev]
            comp = max(comp, float(dev[~cov].max()) if (~cov).any() else 0.0)
            covd = max(covd, float(dev[cov].max()) if cov.any() else 0.0)
        accuracy = {"linf_rel_vs_fp64_reference_composite": comp, "linf_rel_vs_fp64_reference_covered": covd,
                    "fp64_refinement_steps": n_iter,
                    "fp64_reference_vcycles": len(meta["residual_history"]) - 1,
                    "sampled": not meta["full"]}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and bicg:
        t = cpu_reference_bicgstab(meta, wl, 1)
        if t:
            solve_s = t[1] + (n_iter - 1) * (t[2] - t[1])
            cpu = {"value": 1.0 / solve_s, "unit": "solves/s", "cores": 1, "kind": "reference",
                   "sample": f"one single-thread reference BiCGStab solve capped at 1 and at 2 iterations, "
                             f"extrapolated to {n_iter} iterations"}
    elif rank == 0 and world == 1 and not args.no_cpu_baseline:
        res = cpu_reference(meta, 1, 1)
        if res:
            cpu = {"value": res["per_step"][0], "unit": "solves/s", "cores": 1, "kind": "reference",
                   "sample": f"one single-thread reference solve capped at 2 of {res['n_iter']} V-cycles, "
                             f"extrapolated to the full solve (set-up + first + (n-1) x later V-cycle)"}
    cpu_all = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not bicg:
        cpu_all = cpu_reference_openmp(meta, os.cpu_count() or 1)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
            "config": {"workload": wl["name"], "global_batch": world, "cells": sum(ncells),
                       "levels": len(ncells), "boxes": [len(b) for b in meta["boxes"]],
                       ("bicgstab_iterations_per_solve" if bicg else "vcycles_per_solve"): n_iter,
                       "l2": "working set > L2 (no flush)",
                       "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU",
                       "cuda_graphs": not args.no_graphs},
            "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
            "roofline": roofline, "vcycle": vcycle, "breakdown": breakdown, "cpu_baseline": cpu,
            "cpu_baseline_all_cores": cpu_all, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches, "launch_index_at_timed_start": launches0,
            "relax_variants": h.relax_variants(),
        }
        if accuracy:
            line["accuracy"] = accuracy
    h.close()
    if rank == 0:
        if world == 1 and args.workload == "config1" and args.extras:
            line["extra_workloads"] = extra_workloads(args, cmg)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
