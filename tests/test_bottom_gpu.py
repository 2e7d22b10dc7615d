"""The bottom solve (BiCGStabSolver or RelaxSolver on the deepest multigrid
level) run by one thread block and run across the whole device in one
cooperative launch gives the same bits: both sum every dot product and norm
box by box in the reference's order, and both read a face ghost from the
cell its exchange or boundary condition copies.  A single hierarchy whose
bottom level has 4096 cells or more takes the grid-wide solve by itself; the
fixtures with 4096 boxes of 4^3 (bottom level 32^3 in 4096 boxes of 2^3, the
bottom of the 512^3 periodic configuration in 32^3 boxes) reproduce the
reference solve bit for bit through it."""
import numpy as np
import pytest

from conftest import golden


def make(cmg, name):
    meta, arrays = golden(name)
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"],
                      bc=meta.get("bc"))
    h.fill_synthetic(meta["seed"])
    p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                         eps=meta["eps"], hang=meta["hang"])
    return h, p, meta, arrays


def check_reference(h, out, meta, arrays):
    assert out["exit_status"] == meta["exit_status"]
    assert np.array_equal(out["history"], np.array(meta["residual_history"]))
    for lev in range(len(meta["boxes"])):
        phi = h.phi(lev)
        ref = arrays[f"phi{lev}"] if meta["full"] else arrays[f"phi{lev}_sample"]
        got = phi if meta["full"] else phi[::meta["sample_stride"]]
        assert np.array_equal(got, ref), lev


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["helmholtz_1lev_64_periodic_box4", "vc_1lev_64_box4"])
def test_large_bottom_runs_on_the_grid_and_matches_reference(cmg, name):
    h, p, meta, arrays = make(cmg, name)
    assert h.set_bottom_grid(-1)
    check_reference(h, h.solve(p), meta, arrays)
    assert not h.set_bottom_grid(0)
    check_reference(h, h.solve(p), meta, arrays)
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["vc_3lev_16", "poisson_3lev_16_walls", "helmholtz_1lev_32_ppnndd",
                                  "vc_1lev_32_periodic", "helmholtz_1lev_64_periodic_box4"])
def test_grid_and_block_bottoms_are_bit_identical(cmg, name):
    """BiCGStab and RelaxSolver bottoms, norm types 2 and 0, FP64 and mixed V-cycles, launched and graph-replayed."""
    h, p, meta, arrays = make(cmg, name)
    nlev = len(meta["boxes"])
    for kind, norm in ((0, 2), (0, 0), (1, 2), (1, 0)):
        h.set_bottom_solver(kind=kind, norm_type=norm)
        for mixed in (False, True):
            ref = None
            for mode, graphs in ((0, False), (1, False), (1, True), (0, True)):
                assert h.set_bottom_grid(mode) == (mode == 1)
                h.use_graphs(graphs)
                out = h.solve(p, mixed=mixed)
                got = (out["exit_status"], out["history"].tolist(), [h.phi(l).tobytes() for l in range(nlev)])
                ref = ref or got
                assert got == ref, (kind, norm, mixed, mode, graphs)
            if kind == 0 and norm == 2 and not mixed:
                check_reference(h, out, meta, arrays)
    h.close()


@pytest.mark.gpu
def test_forest_keeps_one_block_per_hierarchy(cmg):
    meta, _ = golden("vc_3lev_16")
    f = cmg.Forest(meta["n0"], [meta["boxes"]] * 2, op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
    assert not f.set_bottom_grid(1)
    f.close()
