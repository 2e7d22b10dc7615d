"""cmg_residual_norm_noalloc: the composite residual max-norm with its
reduction scratch in a fixed device array of the library, allocating no
memory.  It must return the value cmg_residual_norm returns (a maximum does
not depend on reduction order, so the two agree to the last bit; the test
allows 1e-14 relative), on two calls in a row, and leave the device's free
memory unchanged.  The file is named to be collected last, so it runs both
after the other GPU tests and, on its own, in a fresh process."""
import numpy as np
import pytest

from conftest import golden

TOL = 1e-14


def hierarchy(cmg, name):
    meta, _ = golden(name)
    h = cmg.Hierarchy(meta["n0"], meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"], bc=meta.get("bc"))
    h.fill_synthetic(meta["seed"])
    return h, meta


def close(a, b):
    return abs(a - b) <= TOL * max(abs(a), abs(b))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["poisson_1lev_32", "poisson_3lev_16", "vc_3lev_16", "helmholtz_2lev_16"])
def test_matches_residual_norm_twice(cmg, name):
    h, meta = hierarchy(cmg, name)
    # phi = 0: the residual is the right-hand side on uncovered cells.
    ref = h.residual_norm()
    n1 = h.residual_norm_noalloc()
    n2 = h.residual_norm_noalloc()
    assert ref > 0
    assert close(n1, ref) and close(n2, ref), (n1, n2, ref)
    # A partly converged phi exercises the coarse-fine and reflux terms.
    p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=2,
                         eps=meta["eps"], hang=meta["hang"])
    h.solve(p)
    ref = h.residual_norm()
    n1 = h.residual_norm_noalloc()
    n2 = h.residual_norm_noalloc()
    assert close(n1, ref) and close(n2, ref), (n1, n2, ref)
    h.close()


@pytest.mark.gpu
def test_leaves_free_memory_unchanged(cmg):
    import torch

    h, _ = hierarchy(cmg, "vc_3lev_16")
    first = h.residual_norm_noalloc()  # first call on the device: scratch lookup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    vals = [h.residual_norm_noalloc() for _ in range(5)]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert all(v == first for v in vals)
    h.close()


@pytest.mark.gpu
def test_rejects_level_beyond_scratch(cmg):
    # 34^3 domain in 2^3 boxes: 17^3 = 4913 boxes on level 0, above the
    # 4096 per-level partials the static scratch holds.
    n0 = 34
    boxes = [(i, j, k, i + 1, j + 1, k + 1) for k in range(0, n0, 2) for j in range(0, n0, 2)
             for i in range(0, n0, 2)]
    h = cmg.Hierarchy(n0, [boxes], op=0, alpha=0.0, beta=1.0)
    with pytest.raises(cmg.CmgError) as err:
        h.residual_norm_noalloc()
    assert err.value.code == cmg.CMG_EINVAL
    assert "4096" in str(err.value)
    # The rejected call launched nothing; the ordinary entry point still works.
    assert np.isfinite(h.residual_norm())
    h.close()


@pytest.mark.gpu
def test_forgotten_scratch_is_looked_up_again(cmg):
    """cmg_residual_norm_noalloc_forget drops the cached scratch address (for a caller that reset the device);
    the next call looks it up again and gives the same value."""
    h, _ = hierarchy(cmg, "vc_3lev_16")
    before = h.residual_norm_noalloc()
    assert cmg.lib().cmg_residual_norm_noalloc_forget() == cmg.CMG_OK
    assert h.residual_norm_noalloc() == before
    h.close()
