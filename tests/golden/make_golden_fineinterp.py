"""Regenerates the FineInterp fixtures (fineinterp_*.json|npz) from the reference oracle.

oracle/_ref/cmg_oracle_fineinterp runs the reference's FineInterp
(AMRTools/FineInterp.cpp, default PCInterp boundary limiting, or
pwcinterpToFine) compiled from the reference's own sources (oracle/Makefile),
on the hierarchy of an existing AMRMultiGrid fixture.  The coarse data are
either that level's seeded right-hand side ("rhs") or a seeded field with
smooth parts, a jump and noise ("field", stored in the fixture), so that the
limiter takes all of its branches.  Each fixture records the fine level's
valid cells (every `sample_stride`-th).

    python tests/golden/make_golden_fineinterp.py [case ...]
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_fineinterp")

# name: (base fixture, fine level, pwc, input, sample stride); a stride above
# one also leaves the coarse field out of the fixture (the tests rebuild it
# with seeded_field and check its recorded sum)
CASES = {
    "fineinterp_poisson_3lev_32_l1": ("poisson_3lev_32", 1, 0, "rhs", 5),
    "fineinterp_poisson_3lev_32_l2_field": ("poisson_3lev_32", 2, 0, "field", 13),
    "fineinterp_vc_3lev_16_l2_field": ("vc_3lev_16", 2, 0, "field", 3),
    "fineinterp_vc_3lev_16_l1_pwc": ("vc_3lev_16", 1, 1, "field", 1),
    "fineinterp_helmholtz_2lev_16_l1_field": ("helmholtz_2lev_16", 1, 0, "field", 1),
    "fineinterp_config1_vc_3lev_128_l2": ("config1_vc_3lev_128", 2, 0, "rhs", 997),
    "fineinterp_config1_vc_3lev_128_l1_field": ("config1_vc_3lev_128", 1, 0, "field", 211),
}


def cell_indices(boxes):
    """(i, j, k) of every valid cell, per box in order, x fastest."""
    out = []
    for b in boxes:
        k, j, i = np.meshgrid(np.arange(b[2], b[5] + 1), np.arange(b[1], b[4] + 1), np.arange(b[0], b[3] + 1),
                              indexing="ij")
        out.append(np.stack([i.ravel(), j.ravel(), k.ravel()]))
    return np.concatenate(out, axis=1)


def seeded_field(boxes, n, seed):
    """Smooth waves, a jump across a tilted plane and small noise on a level of n^3 cells."""
    i, j, k = cell_indices(boxes).astype(np.float64)
    x, y, z = (i + 0.5) / n, (j + 0.5) / n, (k + 0.5) / n
    f = np.sin(2 * np.pi * x) * np.cos(3 * np.pi * y) + 0.5 * z * z
    f += np.where(x + 0.5 * y + 0.25 * z > 0.9, 1.0, 0.0)
    f += 0.02 * np.random.default_rng(seed).standard_normal(f.size)
    return f


def run_case(name):
    base, level, pwc, inp, stride = CASES[name]
    bmeta = json.load(open(os.path.join(HERE, base + ".json")))
    tmp = os.path.join("/tmp", "cmg_golden_" + name)
    cmd = [ORACLE] + bmeta["args"].split() + [f"level={level}", f"pwc={pwc}", "out=" + tmp]
    arrays, extra = {}, {}
    if inp == "field":
        coarse = seeded_field(bmeta["boxes"][level - 1], bmeta["n0"] << (level - 1), 1000 + level)
        coarse.tofile(tmp + ".coarse")
        cmd.append("coarse=" + tmp + ".coarse")
        if stride == 1:
            arrays["coarse"] = coarse
        extra["coarse_sum"] = float(np.sum(coarse))
    subprocess.run(cmd, check=True)
    meta = json.load(open(tmp + ".json"))
    assert meta["coarse_boxes"] == bmeta["boxes"][level - 1] and meta["fine_boxes"] == bmeta["boxes"][level], \
        "hierarchy differs from the base fixture"
    fine = np.fromfile(tmp + ".bin", dtype=np.float64)
    n = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in meta["fine_boxes"])
    assert fine.size == n
    arrays["fine"] = fine[::stride].copy()
    out = {"base": base, "level": level, "pwc": pwc, "input": inp, "sample_stride": stride, "fine_cells": int(n),
           "fine_absmax": float(np.abs(fine).max()), **extra}
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(out, f, indent=1)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(name, n, out["fine_absmax"])


if __name__ == "__main__":
    for c in sys.argv[1:] or list(CASES):
        run_case(c)
