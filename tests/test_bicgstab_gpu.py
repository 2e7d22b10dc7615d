"""BiCGStab over MultilevelLinearOp preconditioned by AMR multigrid
(cmg_solve_multilevel_bicgstab) against the reference's own
BiCGStabSolver<Vector<LevelData<FArrayBox>*>> solve (fixtures bicgstab_*,
from oracle/_ref/cmg_oracle_mlbicgstab): same hierarchy and seeded inputs as
the base AMRMultiGrid fixture, same solver parameters.  Exit status and
iteration count must match exactly, the initial and final residual norms to
1e-12 of the initial residual, phi to 1e-12 relative L-infinity per level.
Dot products follow the reference's summation order, so single-level solves
must be bit-identical in phi and both residuals."""
import numpy as np
import pytest

from conftest import golden

TOL = 1e-12
CASES = ["bicgstab_poisson_1lev_32", "bicgstab_vc_1lev_32", "bicgstab_helmholtz_2lev_16", "bicgstab_vc_3lev_16",
         "bicgstab_poisson_3lev_32", "bicgstab_config1_vc_3lev_128"]


def params(cmg, meta):
    kv = dict(a.split("=") for a in meta["solver_args"].split())
    return cmg.mlsolve_params(mg_iters=int(kv["mgiters"]), mg_smooth=int(kv["mgsmooth"]), imax=int(kv["imax"]),
                              eps=float(kv["eps"]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_bicgstab_matches_reference(cmg, name):
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    h = cmg.Hierarchy(base["n0"], base["boxes"], op=base["op"], alpha=base["alpha"], beta=base["beta"], bc=base.get("bc"))
    h.fill_synthetic(base["seed"])
    out = h.solve_bicgstab(params(cmg, meta))
    r0 = meta["initial_residual"]
    assert out["exit_status"] == meta["exit_status"]
    assert out["iterations"] == meta["iterations"]
    assert abs(out["initial_residual"] - r0) <= TOL * r0
    assert abs(out["final_residual"] - meta["final_residual"]) <= TOL * r0, (out["final_residual"],
                                                                             meta["final_residual"])
    single = len(base["boxes"]) == 1
    if single:
        assert out["initial_residual"] == r0 and out["final_residual"] == meta["final_residual"]
    stride = meta["sample_stride"]
    for lev in range(len(base["boxes"])):
        ref = arrays[f"phi{lev}"]
        got = h.phi(lev)[::stride]
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(got - ref)) <= TOL * scale, (lev, np.max(np.abs(got - ref)) / scale)
        if single:
            assert np.array_equal(got, ref)
    h.close()


@pytest.mark.gpu
def test_bicgstab_from_current_phi(cmg):
    """zero_phi=False starts from the phi in place: a converged phi converges again at once."""
    meta, _ = golden("bicgstab_vc_3lev_16")
    base, _ = golden(meta["base"])
    h = cmg.Hierarchy(base["n0"], base["boxes"], op=base["op"], alpha=base["alpha"], beta=base["beta"], bc=base.get("bc"))
    h.fill_synthetic(base["seed"])
    p = params(cmg, meta)
    first = h.solve_bicgstab(p)
    again = h.solve_bicgstab(p, zero_phi=False)
    assert again["initial_residual"] <= 2 * first["final_residual"]
    h.close()


@pytest.mark.gpu
def test_bicgstab_graph_replay_is_bit_identical(cmg):
    """Each preconditioner call replayed from a captured CUDA graph gives the same bits as launching it."""
    meta, _ = golden("bicgstab_vc_3lev_16")
    base, _ = golden(meta["base"])
    h = cmg.Hierarchy(base["n0"], base["boxes"], op=base["op"], alpha=base["alpha"], beta=base["beta"], bc=base.get("bc"))
    h.fill_synthetic(base["seed"])
    p = params(cmg, meta)
    plain = h.solve_bicgstab(p)
    phi = [h.phi(l) for l in range(len(base["boxes"]))]
    h.use_graphs(True)
    for _ in range(2):  # capture, then replay
        g = h.solve_bicgstab(p)
        assert g["iterations"] == plain["iterations"] and g["final_residual"] == plain["final_residual"]
        assert np.array_equal(g["history"], plain["history"])
        for l in range(len(phi)):
            assert np.array_equal(h.phi(l), phi[l])
    h.close()
