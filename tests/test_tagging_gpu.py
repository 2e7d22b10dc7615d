"""Device-side tagging (cmg_synthetic_hierarchy_device): the tagging pass of
the example drivers' grid generation (|rhs| at every cell, max-reduction,
threshold, one-cell growth clipped to the domain) runs on the GPU and feeds
the host's Berger-Rigoutsos.  The box lists must be the reference's on every
golden fixture (recorded from the reference's own BRMeshRefine) and the host
path's on a sweep of other parameters; a request served with device tags
gives the same phi bits as one served with host tags."""
import json
import os

import pytest

from conftest import GOLDEN, OTHER_PATHS

FIXTURES = sorted(f[:-5] for f in os.listdir(GOLDEN) if f.endswith(".json") and not f.startswith(OTHER_PATHS))

SWEEP = [
    dict(n0=48, levels=3, maxbox=16, block=8, fill=0.75, seed=7, thresh=0.1),
    dict(n0=64, levels=3, maxbox=16, block=4, fill=0.6, seed=20261204, thresh=0.05),
    dict(n0=32, levels=2, maxbox=32, block=8, fill=0.9, seed=11, thresh=0.2),
    dict(n0=80, levels=2, maxbox=40, block=8, fill=0.5, seed=3, thresh=0.1),
    dict(n0=96, levels=3, maxbox=32, block=8, fill=0.75, seed=20261210, thresh=0.1),
    dict(n0=128, levels=3, maxbox=32, block=8, fill=0.7, seed=5, thresh=0.3),
    dict(n0=16, levels=4, maxbox=8, block=2, fill=0.8, seed=99, thresh=0.0),
    dict(n0=256, levels=2, maxbox=32, block=8, fill=0.75, seed=20261203, thresh=0.1),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_device_tags_match_reference_fixture(cmg, name):
    m = json.load(open(os.path.join(GOLDEN, name + ".json")))
    got = cmg.synthetic_hierarchy(m["n0"], m["levels"], m["maxbox"], m["block"], m["fill"], m["seed"], m["thresh"],
                                  device_tags=True)
    assert got == [[tuple(b) for b in lev] for lev in m["boxes"]]


@pytest.mark.gpu
@pytest.mark.parametrize("case", SWEEP, ids=lambda c: "n{n0}_l{levels}_m{maxbox}_b{block}_t{thresh}".format(**c))
def test_device_tags_match_host_tags(cmg, case):
    args = (case["n0"], case["levels"], case["maxbox"], case["block"], case["fill"], case["seed"], case["thresh"])
    host = cmg.synthetic_hierarchy(*args)
    dev = cmg.synthetic_hierarchy(*args, device_tags=True)
    assert dev == host
    assert len(dev) == case["levels"] or case["thresh"] > 0


@pytest.mark.gpu
def test_served_request_same_with_device_tags(cmg):
    base = dict(n0=48, levels=3, max_box=16, block_factor=8, seed=41, op=1, alpha=1.0, beta=-1.0, mixed=False,
                eps=1e-10)
    reqs = [dict(base, device_tags=False), dict(base, device_tags=True)]
    res, _ = cmg.serve(reqs, max_inflight=2, open_loop=False)
    assert all(r["error"] == 0 for r in res)
    assert res[0]["phi_hash"] == res[1]["phi_hash"]
    assert res[0]["iterations"] == res[1]["iterations"] and res[0]["cells"] == res[1]["cells"]
