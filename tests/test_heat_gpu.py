"""Heat solvers against the reference's (fixtures heat_*, from
oracle/_ref/cmg_oracle_heat): backward Euler (cmg_backward_euler: each step
forms a*phi + dt*src, sets alpha = 1, beta = -dt on every operator with
cmg_set_alpha_beta and solves from the previous phi) and TGA (cmg_tga: two
operator applications and two Helmholtz solves per step).  Every solve's
V-cycle count and exit status must match, and the final phi agree to 1e-12
relative L-infinity per level; single-level runs are bit-identical."""
import numpy as np
import pytest

from conftest import golden

TOL = 1e-12
CASES = ["heat_poisson_1lev_32", "heat_poisson_3lev_16", "heat_vc_3lev_16", "heat_tga_poisson_1lev_32",
         "heat_tga_poisson_3lev_16", "heat_tga_vc_3lev_16"]


def setup(cmg, name):
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    kv = dict(a.split("=") for a in meta["heat_args"].split())
    h = cmg.Hierarchy(base["n0"], base["boxes"], op=int(kv["op"]), alpha=float(kv["alpha"]),
                      beta=float(kv["beta"]))
    h.fill_synthetic(base["seed"])
    for lev in range(len(base["boxes"])):
        h.set_phi(lev, h.get_rhs(lev))  # initial state = the seeded right-hand side, which is also the source
    return h, meta, arrays, base, float(kv["dt"]), int(kv["steps"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_backward_euler_matches_reference(cmg, name):
    h, meta, arrays, base, dt, steps = setup(cmg, name)
    p = cmg.solve_params(pre=4, post=4, bottom=4, iter_max=100, eps=1e-10, hang=1e-10)
    if meta.get("scheme") == "tga":
        out = h.tga(p, dt, steps)
        # the reference records the exit status after each step's second solve
        assert [o["exit_status"] for o in out[1::2]] == meta["exit_status"]
    else:
        out = h.backward_euler(p, dt, steps)
        assert [o["exit_status"] for o in out] == meta["exit_status"]
    assert [o["iterations"] for o in out] == meta["iterations"]
    single = len(base["boxes"]) == 1
    for lev in range(len(base["boxes"])):
        ref = arrays[f"phi{lev}"]
        got = h.phi(lev)
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(got - ref)) <= TOL * scale, (lev, np.max(np.abs(got - ref)) / scale)
        if single:
            assert np.array_equal(got, ref)
    h.close()


@pytest.mark.gpu
def test_set_alpha_beta_matches_a_fresh_hierarchy(cmg):
    """setAlphaAndBeta on a VC hierarchy recomputes lambda everywhere: solving then equals solving on a hierarchy
    created with those coefficients."""
    meta, _ = golden("vc_3lev_16")
    p = cmg.solve_params(pre=4, post=4, bottom=4, iter_max=100, eps=1e-10, hang=1e-10)
    a = cmg.Hierarchy(meta["n0"], meta["boxes"], op=1, alpha=1.0, beta=-1.0)
    a.fill_synthetic(meta["seed"])
    a.set_alpha_beta(2.0, 0.5)
    ra = a.solve(p)
    b = cmg.Hierarchy(meta["n0"], meta["boxes"], op=1, alpha=2.0, beta=0.5)
    b.fill_synthetic(meta["seed"])
    rb = b.solve(p)
    assert np.array_equal(ra["history"], rb["history"])
    for lev in range(len(meta["boxes"])):
        assert np.array_equal(a.phi(lev), b.phi(lev))
    a.close()
    b.close()


@pytest.mark.gpu
def test_tga_graph_replay_is_bit_identical(cmg):
    """With CUDA graphs on, the TGA solves switch between graphs captured per (alpha, beta): same bits as launched."""
    runs = []
    for graphs in (False, True):
        h, meta, arrays, base, dt, steps = setup(cmg, "heat_tga_vc_3lev_16")
        h.use_graphs(graphs)
        p = cmg.solve_params(pre=4, post=4, bottom=4, iter_max=100, eps=1e-10, hang=1e-10)
        out = h.tga(p, dt, 3)
        runs.append(([o["iterations"] for o in out], [h.phi(l) for l in range(len(base["boxes"]))]))
        h.close()
    assert runs[0][0] == runs[1][0]
    for a, b in zip(runs[0][1], runs[1][1]):
        assert np.array_equal(a, b)
