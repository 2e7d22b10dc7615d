"""Grid generation (cmg_synthetic_hierarchy): domainSplit for the base level
and MeshRefine::regrid with Berger-Rigoutsos clustering for the finer ones,
driven by the example drivers' tagging loop.  The box lists must be
identical to the reference's: against every golden fixture (recorded from the
reference's own BRMeshRefine), and, where the oracle is built, against fresh
reference runs with other parameters (block factor, max box, fill ratio,
threshold, seed)."""
import json
import os
import subprocess

import pytest

from conftest import GOLDEN, OTHER_PATHS, ROOT

ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle")
FIXTURES = sorted(f[:-5] for f in os.listdir(GOLDEN) if f.endswith(".json") and not f.startswith(OTHER_PATHS))


@pytest.mark.parametrize("name", FIXTURES)
def test_boxes_match_reference_fixture(cmg, name):
    m = json.load(open(os.path.join(GOLDEN, name + ".json")))
    got = cmg.synthetic_hierarchy(m["n0"], m["levels"], m["maxbox"], m["block"], m["fill"], m["seed"], m["thresh"])
    assert got == [[tuple(b) for b in lev] for lev in m["boxes"]]


EXTRA = [
    dict(n0=48, levels=3, maxbox=16, block=8, fill=0.75, seed=7, thresh=0.1),
    dict(n0=64, levels=3, maxbox=16, block=4, fill=0.6, seed=20261204, thresh=0.05),
    dict(n0=32, levels=2, maxbox=32, block=8, fill=0.9, seed=11, thresh=0.2),
    dict(n0=80, levels=2, maxbox=40, block=8, fill=0.5, seed=3, thresh=0.1),
]


@pytest.mark.skipif(not os.path.exists(ORACLE), reason="oracle not built (needs the reference tree)")
@pytest.mark.parametrize("case", EXTRA, ids=lambda c: "n{n0}_l{levels}_m{maxbox}_b{block}_f{fill}_t{thresh}".format(**c))
def test_boxes_match_fresh_reference_run(cmg, tmp_path, case):
    out = str(tmp_path / "r")
    args = [f"{k}={v}" for k, v in case.items()] + ["op=0", "alpha=0", "beta=1", "iters=1", "out=" + out]
    subprocess.run([ORACLE] + args, check=True, capture_output=True, timeout=600)
    ref = json.load(open(out + ".json"))["boxes"]
    got = cmg.synthetic_hierarchy(case["n0"], case["levels"], case["maxbox"], case["block"], case["fill"],
                                  case["seed"], case["thresh"])
    assert got == [[tuple(b) for b in lev] for lev in ref]
