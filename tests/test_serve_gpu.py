"""The request loop (cmg_serve): many independent solves admitted against a
device-memory budget, each on its own stream, overlapping on the device.
Every result must be the same alone and in the mix -- bit-identical phi
(hash of every valid cell on every level), iteration count and final
residual -- and a served request must reproduce the reference solve of the
same seeded problem."""
import ctypes

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
def test_admission_keeps_the_budget(cmg):
    """A budget that fits the largest request alone: the admitted estimates never add up to more than the
    budget at any moment (a request waits for earlier ones to release theirs), and all finish."""
    alone = [cmg.serve([r], max_inflight=1, open_loop=False)[0][0] for r in MIX[:4]]
    est = [a["estimate_bytes"] for a in alone]
    budget = float(max(est))
    res, _ = cmg.serve(MIX[:4], hbm_budget=budget, max_inflight=4, open_loop=False)
    assert all(r["error"] == 0 and r["exit_status"] & 1 for r in res), res
    events = sorted([(r["admitted"], e) for r, e in zip(res, est)] + [(r["finished"], -e) for r, e in zip(res, est)],
                    key=lambda t: (t[0], t[1]))
    held = 0
    for _, d in events:
        held += d
        assert held <= budget + 1, (held, budget)


@pytest.mark.gpu
def test_failing_requests_leave_the_others_unchanged(cmg):
    """Host fault injection in the request stream: a NaN in a right-hand side (the solve stops with a non-finite
    norm), an invalid description, a request larger than the whole memory budget, one cancelled before it
    starts, one cancelled after two iterations, one whose time limit has passed.  Each fails with its own
    status and a message; every good request in the same run gets the bit-identical result it gets alone."""
    good = MIX[:4]
    alone = [cmg.serve([r], max_inflight=1, open_loop=False)[0][0] for r in good]
    budget = float(sum(a["estimate_bytes"] for a in alone)) * 1.5
    cancelled = ctypes.c_int(1)
    bad = [
        (dict(good[0], inject_nan_rhs=True), cmg.CMG_EDIVERGED),
        (dict(good[1], n0=30, block_factor=8), cmg.CMG_EINVAL),
        (dict(n0=256, levels=3, max_box=32, op=1, alpha=1.0, beta=-1.0, seed=7, mixed=True), cmg.CMG_ENOMEM),
        (dict(good[2], cancel=cancelled), cmg.CMG_ECANCELLED),
        (dict(good[3], inject_cancel_after=2), cmg.CMG_ECANCELLED),
        (dict(good[0], timeout=1e-9), cmg.CMG_ETIMEOUT),
    ]
    reqs = []
    for i in range(max(len(good), len(bad))):
        if i < len(bad):
            reqs.append(bad[i][0])
        if i < len(good):
            reqs.append(good[i])
    res, _ = cmg.serve(reqs, hbm_budget=budget, max_inflight=5, open_loop=False)
    k = 0
    for i in range(max(len(good), len(bad))):
        if i < len(bad):
            r, code = res[k], bad[i][1]
            assert r["error"] == code, (i, r)
            assert r["message"], r
            if code == cmg.CMG_EDIVERGED:
                assert not np.isfinite(r["rfinal"]), r
            if i == 4:
                assert r["iterations"] == 2, r
            k += 1
        if i < len(good):
            r, a = res[k], alone[i]
            assert r["error"] == 0, r
            assert r["phi_hash"] == a["phi_hash"] and r["iterations"] == a["iterations"], (r, a)
            k += 1


@pytest.mark.gpu
def test_nan_right_hand_side_reports_divergence(cmg):
    """cmg_solve on a right-hand side holding a NaN: the max norm propagates the NaN (it is not dropped as a
    max over doubles would), the solve stops with CMG_EDIVERGED and writes its outputs."""
    meta, _ = golden("vc_3lev_16")
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"], bc=meta.get("bc"))
    h.fill_synthetic(meta["seed"])
    rhs = h.get_rhs(2)
    rhs[len(rhs) // 2] = np.nan
    h.set_rhs(2, rhs)
    assert np.isnan(h.residual_norm())
    out = h.solve(cmg.solve_params())
    assert out["diverged"] and out["iterations"] == 0
    assert np.isnan(out["history"][0])
    h.close()


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


BATCH = [
    # one class (same recipe, operator, precision, parameters), different seeds and tolerances
    dict(n0=32, levels=2, max_box=16, op=0, alpha=0.0, beta=1.0, seed=201, mixed=True, eps=1e-10),
    dict(n0=32, levels=2, max_box=16, op=0, alpha=0.0, beta=1.0, seed=202, mixed=True, eps=1e-8),
    dict(n0=32, levels=2, max_box=16, op=0, alpha=0.0, beta=1.0, seed=203, mixed=True, eps=1e-10),
    # another class
    dict(n0=48, levels=2, max_box=24, op=1, alpha=1.0, beta=-1.0, seed=204, mixed=False, eps=1e-10),
    dict(n0=48, levels=2, max_box=24, op=1, alpha=1.0, beta=-1.0, seed=205, mixed=False, eps=1e-8),
    # a class of one
    dict(n0=64, levels=1, max_box=32, op=0, alpha=1.0, beta=-1.0, seed=206, mixed=True, eps=1e-10),
]


@pytest.mark.gpu
def test_batched_requests_give_their_own_results(cmg):
    """cmg_serve_batched: requests of one class in flight together are solved as one forest, each with its own
    tolerance; every result (phi hash, iterations, final norm, exit status) is the one the request gets alone,
    and the batch sizes show that the classes were batched."""
    alone = [cmg.serve([r], max_inflight=1, open_loop=False)[0][0] for r in BATCH]
    for a in alone:
        assert a["error"] == 0 and a["exit_status"] & 1, a
    res, _ = cmg.serve(BATCH, max_inflight=len(BATCH), open_loop=False, batch_window=0.5, max_batch=8)
    for a, b in zip(alone, res):
        assert b["error"] == 0, b
        assert b["phi_hash"] == a["phi_hash"], (a, b)
        assert (b["iterations"], b["exit_status"], b["rfinal"]) == (a["iterations"], a["exit_status"], a["rfinal"])
    assert [b["batch_size"] for b in res] == [3, 3, 3, 2, 2, 1], [b["batch_size"] for b in res]


@pytest.mark.gpu
def test_failures_inside_a_batch_stay_with_their_request(cmg):
    """A NaN right-hand side and a cancellation after two iterations inside one batch: those two members fail
    with their own status, the others in the same forest keep their own results."""
    base = dict(n0=32, levels=2, max_box=16, op=0, alpha=0.0, beta=1.0, mixed=True, eps=1e-10)
    reqs = [dict(base, seed=301), dict(base, seed=302, inject_nan_rhs=True), dict(base, seed=303),
            dict(base, seed=304, inject_cancel_after=2)]
    alone = [cmg.serve([r], max_inflight=1, open_loop=False)[0][0] for r in (reqs[0], reqs[2])]
    res, _ = cmg.serve(reqs, max_inflight=len(reqs), open_loop=False, batch_window=0.5, max_batch=8)
    assert all(r["batch_size"] == 4 for r in res), [r["batch_size"] for r in res]
    assert res[1]["error"] == cmg.CMG_EDIVERGED, res[1]
    assert res[3]["error"] == cmg.CMG_ECANCELLED and res[3]["iterations"] == 2, res[3]
    for a, b in zip(alone, (res[0], res[2])):
        assert b["error"] == 0 and b["phi_hash"] == a["phi_hash"] and b["iterations"] == a["iterations"]
