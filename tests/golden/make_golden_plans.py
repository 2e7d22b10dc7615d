"""Writes the complete Copier plans of the benchmark-size fixtures (whose JSON
keeps only plan sizes) as <case>_plans.npz in this directory, from the
reference's own Copier (oracle/_ref/cmg_oracle plansonly=1, no solve): per
level `exchange<l>` (Copier::exchangeDefine + trimEdges) and, for levels
>= 1, `coarsened_fine<l>` (Copier::define(coarsen(grids[l]), grids[l-1])),
each an int32 array of shape (items, 14): from, to, fromRegion lo/hi,
toRegion lo/hi.

    python tests/golden/make_golden_plans.py [case ...]
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle")

CASES = ["config1_vc_3lev_128", "config2_vc_3lev_256", "helmholtz_1lev_64_periodic_box4", "vc_1lev_64_box4"]


def run_case(name):
    meta = json.load(open(os.path.join(HERE, name + ".json")))
    tmp = os.path.join("/tmp", "cmg_plans_" + name)
    subprocess.run([ORACLE] + meta["args"].split() + ["plansonly=1", "out=" + tmp], check=True)
    raw = np.fromfile(tmp + ".plans", dtype=np.int32)
    arrays, pos = {}, 0
    for lev in range(len(meta["boxes"])):
        for key in (["exchange"] if lev == 0 else ["exchange", "coarsened_fine"]):
            n = int(raw[pos])
            pos += 1
            arrays[f"{key}{lev}"] = raw[pos:pos + 14 * n].reshape(n, 14).copy()
            pos += 14 * n
    assert pos == raw.size, (pos, raw.size)
    np.savez_compressed(os.path.join(HERE, name + "_plans.npz"), **arrays)
    print(name, {k: v.shape[0] for k, v in arrays.items()})


if __name__ == "__main__":
    for n in sys.argv[1:] or CASES:
        run_case(n)
