"""CUDA-graph replay of the solver iteration (cmg_use_graphs): the captured
graph runs the same kernels in the same order as the launched path, so phi
and the residual history are bit-identical, in FP64 and in mixed precision,
and one captured graph serves later solves of the same hierarchy with a new
right-hand side (the bottom solver's metric is read from device memory)."""
import numpy as np
import pytest

from conftest import golden


def make(cmg, name):
    meta, _ = golden(name)
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"], bc=meta.get("bc"))
    h.fill_synthetic(meta["seed"])
    p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                         eps=meta["eps"], hang=meta["hang"])
    return h, p, meta


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["vc_3lev_16", "poisson_3lev_16", "vc_1lev_32"])
@pytest.mark.parametrize("mixed", [False, True])
def test_graph_replay_is_bit_identical(cmg, name, mixed):
    h, p, meta = make(cmg, name)
    nlev = len(meta["boxes"])
    plain = h.solve(p, mixed=mixed)
    phi_plain = [h.phi(l) for l in range(nlev)]
    h.use_graphs(True)
    for _ in range(2):  # capture, then replay
        out = h.solve(p, mixed=mixed)
        assert out["exit_status"] == plain["exit_status"]
        assert np.array_equal(out["history"], plain["history"])
        for l in range(nlev):
            assert np.array_equal(h.phi(l), phi_plain[l])
    # a new right-hand side through the same captured graph
    rhs0 = [h.phi(l) * 0 + 1.0 for l in range(nlev)]
    for l in range(nlev):
        h.set_rhs(l, rhs0[l])
    g = h.solve(p, mixed=mixed)
    phi_g = [h.phi(l) for l in range(nlev)]
    h.use_graphs(False)
    u = h.solve(p, mixed=mixed)
    assert np.array_equal(g["history"], u["history"])
    for l in range(nlev):
        assert np.array_equal(h.phi(l), phi_g[l])
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,num_mg", [("vc_3lev_16", 1), ("poisson_3lev_32", 1), ("helmholtz_2lev_16", 1),
                                         ("vc_3lev_16", 2), ("poisson_1lev_32", 1), ("vc_1lev_32", 2),
                                         ("poisson_3lev_32_walls", 1), ("vc_3lev_16_walls", 2),
                                         ("helmholtz_1lev_32_periodic", 1), ("helmholtz_1lev_32_ppnndd", 2),
                                         ("helmholtz_1lev_64_periodic_box4", 1)])
def test_relaxation_variants_are_bit_identical(cmg, name, num_mg):
    """Ghost fill before each colour pass (mode 1), face ghosts evaluated in
    the pass (mode 2), fused sweeps (mode 3: both colours per launch, boxes
    marching in z, exchange-face colour-1 cells in a second launch) and the
    autotuned mix (mode 0) give the same bits, with V-cycles and with W-cycles
    (num_mg=2), on one and on several levels, FP64 and mixed precision, on
    walled and periodic domains."""
    h, p, meta = make(cmg, name)
    p.num_mg = num_mg
    nlev = len(meta["boxes"])
    ref = None
    for mode in (1, 2, 3, 0):
        h.set_relax_mode(mode)
        for mixed in (False, True):
            out = h.solve(p, mixed=mixed)
            got = (out["history"].tolist(), [h.phi(l).tobytes() for l in range(nlev)])
            if ref is None or mixed not in ref:
                ref = ref or {}
                ref.setdefault(mixed, got)
            assert got == ref[mixed], (mode, mixed)
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["config1_vc_3lev_128", "vc_3lev_32", "poisson_3lev_16_walls"])
def test_fused_sweeps_match_reference(cmg, name):
    """Every level relaxed with fused sweeps (mode 3) reproduces the reference solve bit for bit."""
    meta, arrays = golden(name)
    h, p, _ = make(cmg, name)
    h.set_relax_mode(3)
    out = h.solve(p)
    assert np.array_equal(out["history"], np.array(meta["residual_history"]))
    for lev in range(len(meta["boxes"])):
        phi = h.phi(lev)
        ref = arrays[f"phi{lev}"] if meta["full"] else arrays[f"phi{lev}_sample"]
        got = phi if meta["full"] else phi[::meta["sample_stride"]]
        assert np.array_equal(got, ref), lev
    h.close()
