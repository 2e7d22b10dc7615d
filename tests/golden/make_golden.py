"""Regenerates the golden fixtures in this directory from the reference oracle.

The oracle binary (oracle/_ref/cmg_oracle) is the reference's own
AMRMultiGrid solve compiled from its C++ sources with the C++ restatement of
its ChF kernels (see oracle/Makefile).  Each case records, from the reference:
the box layout of every level (domainSplit + BRMeshRefine), the exchange and
coarsened-fine copier plans, the per-iteration composite residual history,
the exit status, checksums of the right-hand side, and phi (all cells for
small cases, a strided sample for the benchmark-size cases).

    python tests/golden/make_golden.py [--from=<prefix>] [case ...]

(--from reuses an oracle run already written with out=<prefix>.)
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle")

# name: (oracle arguments, store full phi)
CASES = {
    "poisson_1lev_32": ("n0=32 levels=1 maxbox=16 op=0 alpha=0 beta=1", True),
    "helmholtz_1lev_32": ("n0=32 levels=1 maxbox=16 op=0 alpha=1 beta=-1", True),
    "vc_1lev_32": ("n0=32 levels=1 maxbox=16 op=1 alpha=1 beta=-1", True),
    "poisson_3lev_16": ("n0=16 levels=3 maxbox=8 block=4 op=0 alpha=0 beta=1", True),
    "helmholtz_2lev_16": ("n0=16 levels=2 maxbox=8 block=4 op=0 alpha=1 beta=-1", True),
    "vc_3lev_16": ("n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=-1", True),
    "poisson_3lev_32": ("n0=32 levels=3 maxbox=16 op=0 alpha=0 beta=1", False),
    # homogeneous Neumann faces (walls) beside Dirichlet ones (outflow), as the AMRINS projection's pressure BC
    "poisson_3lev_16_walls": ("n0=16 levels=3 maxbox=8 block=4 op=0 alpha=0 beta=1 bc=NNNNND", True),
    "vc_3lev_16_walls": ("n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=-1 bc=NDNDNN", True),
    "helmholtz_2lev_16_neumann": ("n0=16 levels=2 maxbox=8 block=4 op=0 alpha=1 beta=-1 bc=NNNNNN", True),
    "poisson_3lev_32_walls": ("n0=32 levels=3 maxbox=16 op=0 alpha=0 beta=1 bc=NNNNND", False),
    # periodic directions (one-level hierarchies), the published Proto AMRPoisson configuration's operator
    "helmholtz_1lev_32_periodic": ("n0=32 levels=1 maxbox=16 op=0 alpha=1 beta=-0.1 bc=PPPPPP", True),
    "vc_1lev_32_periodic": ("n0=32 levels=1 maxbox=16 op=1 alpha=1 beta=-1 bc=PPPPPP", True),
    "helmholtz_1lev_32_ppnndd": ("n0=32 levels=1 maxbox=16 op=0 alpha=1 beta=-0.1 bc=PPNNDD", True),
    # 4096 boxes of 4^3: the bottom level (32^3 in 4096 boxes of 2^3) is large enough for the grid-wide bottom solve
    "helmholtz_1lev_64_periodic_box4": ("n0=64 levels=1 maxbox=4 block=4 op=0 alpha=1 beta=-0.1 bc=PPPPPP", False),
    "vc_1lev_64_box4": ("n0=64 levels=1 maxbox=4 block=4 op=1 alpha=1 beta=-1", False),
    "vc_3lev_32": ("n0=32 levels=3 maxbox=16 op=1 alpha=1 beta=-1", False),
    "vc_2lev_64": ("n0=64 levels=2 maxbox=32 op=1 alpha=1 beta=-1", False),
    "config0_poisson_64": ("n0=64 levels=1 maxbox=32 op=0 alpha=0 beta=1", True),
    "config1_vc_3lev_128": ("n0=128 levels=3 maxbox=32 op=1 alpha=1 beta=-1", False),
    # the ~40M-cell mixed-precision workload: sparser samples keep the fixture small
    "config2_vc_3lev_256": ("n0=256 levels=3 maxbox=32 op=1 alpha=1 beta=-1", False, 1009),
}
SAMPLE_STRIDE = 97


def run_case(name, args, full, stride=SAMPLE_STRIDE, prefix=None):
    """prefix: reuse an oracle run already written to <prefix>.json/.bin."""
    tmp = prefix or os.path.join("/tmp", "cmg_golden_" + name)
    if not prefix:
        cmd = [ORACLE] + args.split() + ["out=" + tmp]
        subprocess.run(cmd, check=True)
    meta = json.load(open(tmp + ".json"))
    raw = np.fromfile(tmp + ".bin", dtype=np.float64)
    pos = 0
    levels = []
    for lev, boxes in enumerate(meta["boxes"]):
        ncell = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in boxes)
        rhs = raw[pos:pos + ncell]
        pos += ncell
        phi = raw[pos:pos + ncell]
        pos += ncell
        if meta["op"] == 1:
            pos += ncell
            for d in range(3):
                nf = sum((b[3] - b[0] + 1 + (d == 0)) * (b[4] - b[1] + 1 + (d == 1)) * (b[5] - b[2] + 1 + (d == 2))
                         for b in boxes)
                pos += nf
        levels.append((rhs, phi))
    assert pos == raw.size, (pos, raw.size)
    meta["args"] = args
    meta["rhs_sum"] = [float(np.sum(r)) for r, _ in levels]
    meta["phi_absmax"] = [float(np.max(np.abs(p))) for _, p in levels]
    meta["sample_stride"] = stride
    arrays = {}
    for lev, (rhs, phi) in enumerate(levels):
        if full:
            arrays[f"phi{lev}"] = phi
        else:
            arrays[f"phi{lev}_sample"] = phi[::stride].copy()
        arrays[f"rhs{lev}_sample"] = rhs[::stride].copy()
    meta["full"] = full
    if len(json.dumps(meta.get("exchange_plans", []))) > 400000:
        # plans of the big cases are checked through their sizes only
        meta["exchange_plan_sizes"] = [len(p) for p in meta.pop("exchange_plans")]
        meta["coarsened_fine_plan_sizes"] = [len(p) for p in meta.pop("coarsened_fine_plans")]
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(meta, f)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(name, "levels", len(levels), "iters", len(meta["residual_history"]) - 1, "exit", meta["exit_status"])


def main():
    args = sys.argv[1:]
    prefix = None
    if args and args[0].startswith("--from="):
        prefix = args.pop(0)[len("--from="):]
    names = args or list(CASES)
    for n in names:
        run_case(n, *CASES[n], prefix=prefix)


if __name__ == "__main__":
    main()
