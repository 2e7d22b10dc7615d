"""Regenerates the backward-Euler fixtures (heat_*.json|npz) from the reference oracle.

oracle/_ref/cmg_oracle_heat runs the reference's BackwardEuler or AMRTGA heat
solver (lib/src/AMRElliptic/BackwardEuler.cpp, AMRTGA.H, over AMRMultiGrid),
compiled from the reference's own sources (oracle/Makefile), for a few steps:
the initial state and the source are the seeded right-hand side.  Each case uses the hierarchy
of an existing AMRMultiGrid fixture (same grid arguments and seed) with its
own operator coefficients and time step, and records every step's exit
status and V-cycle count and the final phi on every level.

    python tests/golden/make_golden_heat.py [case ...]
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_heat")

# name: (base AMRMultiGrid fixture, operator and stepping arguments)
CASES = {
    "heat_poisson_1lev_32": ("poisson_1lev_32", "op=0 alpha=1 beta=1 dt=1e-3 steps=3"),
    "heat_poisson_3lev_16": ("poisson_3lev_16", "op=0 alpha=1 beta=1 dt=1e-3 steps=3"),
    "heat_vc_3lev_16": ("vc_3lev_16", "op=1 alpha=1 beta=1 dt=1e-6 steps=3"),
    "heat_tga_poisson_1lev_32": ("poisson_1lev_32", "op=0 alpha=1 beta=1 dt=1e-3 steps=2 scheme=tga"),
    "heat_tga_poisson_3lev_16": ("poisson_3lev_16", "op=0 alpha=1 beta=1 dt=1e-3 steps=2 scheme=tga"),
    "heat_tga_vc_3lev_16": ("vc_3lev_16", "op=1 alpha=1 beta=1 dt=1e-6 steps=2 scheme=tga"),
}


def run_case(name):
    base, heat_args = CASES[name]
    bmeta = json.load(open(os.path.join(HERE, base + ".json")))
    grid_args = [a for a in bmeta["args"].split() if not a.split("=")[0] in ("op", "alpha", "beta")]
    tmp = os.path.join("/tmp", "cmg_golden_" + name)
    subprocess.run([ORACLE] + grid_args + heat_args.split() + ["out=" + tmp], check=True)
    meta = json.load(open(tmp + ".json"))
    raw = np.fromfile(tmp + ".bin", dtype=np.float64)
    arrays, pos = {}, 0
    for lev, boxes in enumerate(bmeta["boxes"]):
        n = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in boxes)
        arrays[f"phi{lev}"] = raw[pos:pos + n].copy()
        pos += n
    assert pos == raw.size
    meta["base"] = base
    meta["heat_args"] = heat_args
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(name, meta["exit_status"], meta["iterations"])


if __name__ == "__main__":
    for n in sys.argv[1:] or list(CASES):
        run_case(n)
