"""Device-side synthetic inputs (cmg_fill_synthetic_device, used for served
requests): the same seeded fields and coefficient set-up as the host
generator, evaluated with the CUDA math library, so values agree to within
the last bits of exp and cos, and the solve behaves identically."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["vc_3lev_16", "poisson_3lev_16", "vc_1lev_32"])
def test_device_inputs_match_host_inputs(cmg, name):
    meta, _ = golden(name)
    p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                         eps=meta["eps"], hang=meta["hang"])
    nlev = len(meta["boxes"])
    res = []
    for device in (False, True):
        h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"], bc=meta.get("bc"))
        h.fill_synthetic(meta["seed"], device=device)
        rhs = [h.get_rhs(l) for l in range(nlev)]
        out = h.solve(p)
        res.append((rhs, out, [h.phi(l) for l in range(nlev)]))
        h.close()
    (rh, oh, ph), (rd, od, pd) = res
    for l in range(nlev):
        scale = np.max(np.abs(rh[l]))
        assert np.max(np.abs(rh[l] - rd[l])) <= 1e-14 * scale
        assert np.max(np.abs(ph[l] - pd[l])) <= 1e-12 * np.max(np.abs(ph[l]))
    assert od["exit_status"] == oh["exit_status"] and od["iterations"] == oh["iterations"]
    assert np.max(np.abs(od["history"] - oh["history"])) <= 1e-12 * oh["history"][0]
