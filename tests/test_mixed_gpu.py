"""Mixed precision (cmg_solve_mixed): FP32 AMR V-cycles inside FP64 iterative
refinement, the composite residual with its reflux correction, the bottom
solve and the norms in FP64.  Against the FP64 reference solve of every
golden case: the same exit status and number of iterations (each one FP64
refinement step), the final composite residual below eps * r0, and the
composite solution -- phi on the cells not covered by a finer level -- within
1e-12 relative L-infinity of the reference's FP64 phi.  Coarse cells under a
finer level are not part of the composite solution (the composite residual
is zero there by construction); their FP32 rounding (about 1e-7 relative) is
stated, not bounded tighter."""
import numpy as np
import pytest

from conftest import covered_mask, golden, golden_names

TOL_COMPOSITE = 1e-12
TOL_COVERED = 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name", golden_names())
def test_mixed_matches_fp64_reference(cmg, name):
    meta, arrays = golden(name)
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"], bc=meta.get("bc"))
    h.fill_synthetic(meta["seed"])
    p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                         eps=meta["eps"], hang=meta["hang"])
    out = h.solve(p, mixed=True)
    ref_hist = meta["residual_history"]
    assert out["exit_status"] == meta["exit_status"]
    assert out["iterations"] == len(ref_hist) - 1
    hist = out["history"]
    assert hist[-1] <= meta["eps"] * hist[0]
    nlev = len(meta["boxes"])
    for lev in range(nlev):
        phi = h.phi(lev)
        cov = covered_mask(meta["boxes"][lev], meta["boxes"][lev + 1]) if lev + 1 < nlev else np.zeros(phi.size, bool)
        if meta["full"]:
            ref = arrays[f"phi{lev}"]
        else:
            ref = arrays[f"phi{lev}_sample"]
            phi, cov = phi[::meta["sample_stride"]], cov[::meta["sample_stride"]]
        dev = np.abs(phi - ref) / meta["phi_absmax"][lev]
        assert dev[~cov].max() <= TOL_COMPOSITE, (lev, dev[~cov].max())
        if cov.any():
            assert dev[cov].max() <= TOL_COVERED, (lev, dev[cov].max())
    h.close()
