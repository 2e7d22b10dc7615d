"""The request loop (cmg_serve): many independent solves admitted against a
device-memory budget, each on its own stream, overlapping on the device.
Every result must be the same alone and in the mix -- bit-identical phi
(hash of every valid cell on every level), iteration count and final
residual -- and a served request must reproduce the reference solve of the
same seeded problem."""
import numpy as np
import pytest

from conftest import golden

MIX = [
    dict(n0=32, levels=2, max_box=16, op=0, alpha=0.0, beta=1.0, seed=101, mixed=True),
    dict(n0=48, levels=2, max_box=24, op=1, alpha=1.0, beta=-1.0, seed=102, mixed=True),
    dict(n0=64, levels=1, max_box=32, op=0, alpha=1.0, beta=-1.0, seed=103, mixed=False),
    dict(n0=32, levels=3, max_box=16, op=1, alpha=1.0, beta=-1.0, seed=104, mixed=False),
    dict(n0=64, levels=2, max_box=32, op=1, alpha=1.0, beta=-1.0, seed=105, mixed=True),
    dict(n0=48, levels=1, max_box=16, op=0, alpha=0.0, beta=1.0, seed=106, mixed=True),
]


@pytest.mark.gpu
def test_each_result_is_the_same_alone_and_in_the_mix(cmg):
    alone = [cmg.serve([r], max_inflight=1, open_loop=False)[0][0] for r in MIX]
    for a in alone:
        assert a["error"] == 0 and a["exit_status"] & 1, a
        assert a["rfinal"] <= 1e-10 * a["r0"]
    mixed, wall = cmg.serve(MIX, max_inflight=len(MIX), open_loop=False)
    for a, b in zip(alone, mixed):
        assert b["error"] == 0
        assert b["phi_hash"] == a["phi_hash"]
        assert b["iterations"] == a["iterations"]
        assert b["rfinal"] == a["rfinal"]


@pytest.mark.gpu
def test_tight_budget_admits_one_at_a_time(cmg):
    res, _ = cmg.serve(MIX[:3], hbm_budget=1.0, max_inflight=3, open_loop=False)
    spans = sorted((r["admitted"], r["finished"]) for r in res)
    for (a0, f0), (a1, _) in zip(spans, spans[1:]):
        assert a1 >= f0 - 1e-3  # the next admission waits for the previous release
    assert all(r["error"] == 0 and r["exit_status"] & 1 for r in res)


@pytest.mark.gpu
def test_served_request_reproduces_reference_solve(cmg):
    meta, _ = golden("vc_3lev_16")
    req = dict(n0=meta["n0"], levels=meta["levels"], max_box=meta["maxbox"], block_factor=meta["block"],
               fill_ratio=meta["fill"], thresh=meta["thresh"], seed=meta["seed"], op=meta["op"],
               alpha=meta["alpha"], beta=meta["beta"], mixed=False,
               params=cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"],
                                       iter_max=meta["iters"], eps=meta["eps"], hang=meta["hang"]))
    res, _ = cmg.serve([req], max_inflight=1, open_loop=False)
    r = res[0]
    hist = meta["residual_history"]
    assert r["exit_status"] == meta["exit_status"]
    assert r["iterations"] == len(hist) - 1
    assert abs(r["rfinal"] - hist[-1]) <= 1e-12 * hist[0]
