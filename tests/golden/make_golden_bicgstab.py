"""Regenerates the BiCGStab fixtures (bicgstab_*.json|npz) from the reference oracle.

oracle/_ref/cmg_oracle_mlbicgstab runs the reference's
BiCGStabSolver<Vector<LevelData<FArrayBox>*>> over MultilevelLinearOp
preconditioned by AMR multigrid (the variable-coefficient example's solve
path), compiled from the reference's own sources (oracle/Makefile).  Each case
uses the hierarchy and inputs of an existing AMRMultiGrid fixture (same grid
and problem arguments) and records the exit status, iteration count, initial
and final residual norms, and phi on every level.

    python tests/golden/make_golden_bicgstab.py [case ...]
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_mlbicgstab")

# name: (base AMRMultiGrid fixture, solver arguments, phi sample stride (1: every cell))
CASES = {
    "bicgstab_poisson_1lev_32": ("poisson_1lev_32", "mgiters=1 mgsmooth=4 eps=1e-9 imax=100", 1),
    "bicgstab_vc_1lev_32": ("vc_1lev_32", "mgiters=2 mgsmooth=4 eps=1e-9 imax=100", 1),
    "bicgstab_helmholtz_2lev_16": ("helmholtz_2lev_16", "mgiters=1 mgsmooth=2 eps=1e-10 imax=100", 1),
    "bicgstab_vc_3lev_16": ("vc_3lev_16", "mgiters=2 mgsmooth=4 eps=1e-9 imax=100", 1),
    "bicgstab_poisson_3lev_32": ("poisson_3lev_32", "mgiters=1 mgsmooth=4 eps=1e-9 imax=100", 97),
    # the config-1 hierarchy as the bench's config1-bicgstab workload solves it (about 3 minutes)
    "bicgstab_config1_vc_3lev_128": ("config1_vc_3lev_128", "mgiters=2 mgsmooth=4 eps=1e-10 imax=100", 997),
}


def run_case(name):
    base, solver_args, stride = CASES[name]
    bmeta = json.load(open(os.path.join(HERE, base + ".json")))
    tmp = os.path.join("/tmp", "cmg_golden_" + name)
    cmd = [ORACLE] + bmeta["args"].split() + solver_args.split() + ["out=" + tmp]
    subprocess.run(cmd, check=True)
    meta = json.load(open(tmp + ".json"))
    assert meta["boxes"] == bmeta["boxes"], "hierarchy differs from the base fixture"
    raw = np.fromfile(tmp + ".bin", dtype=np.float64)
    arrays, pos = {}, 0
    for lev, boxes in enumerate(meta["boxes"]):
        n = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in boxes)
        arrays[f"phi{lev}"] = raw[pos:pos + n][::stride].copy()
        pos += n
    assert pos == raw.size
    del meta["boxes"]
    meta["base"] = base
    meta["solver_args"] = solver_args
    meta["sample_stride"] = stride
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(name, meta["exit_status"], meta["iterations"], meta["initial_residual"], meta["final_residual"])


if __name__ == "__main__":
    for n in sys.argv[1:] or list(CASES):
        run_case(n)
