"""Forests (cmg_forest_create / cmg_forest_solve): several hierarchies solved
together, every V-cycle operation one launch over all of their boxes.  Each
hierarchy's result must be the one its own solve gives, bit for bit: exit
status, iteration count, final residual norm and phi, in FP64 and in mixed
precision, with hierarchies that stop at different iterations, and a forest
member built on a golden fixture reproduces the reference's solve."""
import numpy as np
import pytest

from conftest import golden


def spec_boxes(cmg, n0, levels, max_box, seed, block=8):
    return cmg.synthetic_hierarchy(n0, levels, max_box, block, 0.75, seed, 0.1)


def solo(cmg, n0, boxes, op, alpha, beta, seed, params, mixed, device_fill, bc=None):
    h = cmg.Hierarchy(n0, boxes, op=op, alpha=alpha, beta=beta, bc=bc)
    h.fill_synthetic(seed, device=device_fill)
    out = h.solve(params, mixed=mixed)
    phis = [h.phi(l) for l in range(len(boxes))]
    rhs = [h.get_rhs(l) for l in range(len(boxes))]
    h.close()
    return out, phis, rhs


CASES = [
    # n0, levels, max box, op, alpha, beta, seeds, device fill, bc
    (32, 2, 16, 0, 0.0, 1.0, [11, 12, 13, 14], False, None),
    (32, 3, 16, 0, 1.0, -1.0, [21, 22, 23], False, None),
    (48, 2, 24, 1, 1.0, -1.0, [31, 32, 33], True, None),
    (32, 2, 16, 0, 0.0, 1.0, [41, 42, 43], False, "NNNNND"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("mixed", [False, True])
def test_forest_matches_each_solo_solve(cmg, case, mixed):
    n0, levels, max_box, op, alpha, beta, seeds, device_fill, bc = CASES[case]
    params = cmg.solve_params(eps=1e-10)
    hb = [spec_boxes(cmg, n0, levels, max_box, s) for s in seeds]
    ref = [solo(cmg, n0, b, op, alpha, beta, s, params, mixed, device_fill, bc) for b, s in zip(hb, seeds)]
    f = cmg.Forest(n0, hb, op=op, alpha=alpha, beta=beta, bc=bc)
    if device_fill:
        f.fill_synthetic(seeds)
    else:
        for k, r in enumerate(ref):
            for lev in range(len(hb[k])):
                f.set_rhs(k, lev, r[2][lev])
    outs = f.solve(params, mixed=mixed)
    for k, (o, phis, _) in enumerate(ref):
        got = outs[k]
        assert got["exit_status"] == o["exit_status"], (k, got, o["exit_status"])
        assert got["iterations"] == o["iterations"], (k, got, o["iterations"])
        assert got["final_norm"] == o["history"][-1], (k, got, o["history"][-1])
        for lev in range(len(hb[k])):
            assert np.array_equal(f.phi(k, lev), phis[lev]), (k, lev)
    f.close()


@pytest.mark.gpu
def test_forest_member_reproduces_the_reference(cmg):
    """The poisson_3lev_32 fixture's hierarchy solved inside a forest with two other hierarchies gives the
    reference's residual norms and phi."""
    meta, arrays = golden("poisson_3lev_32")
    n0 = meta["n0"]
    others = [spec_boxes(cmg, n0, 3, 16, s) for s in (51, 52)]
    hb = [meta["boxes"]] + others
    solo_h = cmg.Hierarchy(n0, meta["boxes"], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
    solo_h.fill_synthetic(meta["seed"])
    rhs0 = [solo_h.get_rhs(l) for l in range(len(meta["boxes"]))]
    solo_h.close()
    f = cmg.Forest(n0, hb, op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
    for lev in range(len(meta["boxes"])):
        f.set_rhs(0, lev, rhs0[lev])
    for k, s in ((1, 51), (2, 52)):
        h = cmg.Hierarchy(n0, hb[k], op=meta["op"], alpha=meta["alpha"], beta=meta["beta"])
        h.fill_synthetic(s)
        for lev in range(len(hb[k])):
            f.set_rhs(k, lev, h.get_rhs(lev))
        h.close()
    p = cmg.solve_params(pre=meta["pre"], post=meta["post"], bottom=meta["bottom"], iter_max=meta["iters"],
                         eps=meta["eps"], hang=meta["hang"])
    out = f.solve(p)[0]
    assert out["exit_status"] == meta["exit_status"]
    assert out["iterations"] == len(meta["residual_history"]) - 1
    assert out["final_norm"] == meta["residual_history"][-1]
    for lev in range(len(meta["boxes"])):
        got = f.phi(0, lev)
        ref = arrays[f"phi{lev}"] if meta["full"] else arrays[f"phi{lev}_sample"]
        got = got if meta["full"] else got[::meta["sample_stride"]]
        assert np.array_equal(got, ref), lev
    f.close()


@pytest.mark.gpu
def test_forest_refuses_mismatched_hierarchies(cmg):
    a = spec_boxes(cmg, 32, 2, 16, 61)
    b = spec_boxes(cmg, 32, 2, 32, 62)  # another level-0 layout: other multigrid depths
    with pytest.raises(cmg.CmgError):
        cmg.Forest(32, [a, b])


@pytest.mark.gpu
def test_finished_hierarchies_stop_changing(cmg):
    """A member whose solve ends at once (zero right-hand side: norm 0) and one that ends early (a loose
    iteration cap reached first by nobody else is not possible, so a zero and a scaled right-hand side) keep
    the phi of their own solves while the others go on."""
    n0, seeds = 32, [71, 72, 73]
    hb = [spec_boxes(cmg, n0, 2, 16, s) for s in seeds]
    params = cmg.solve_params(eps=1e-10)
    rhs = []
    for b, s in zip(hb, seeds):
        h = cmg.Hierarchy(n0, b)
        h.fill_synthetic(s)
        rhs.append([h.get_rhs(l) for l in range(2)])
        h.close()
    rhs[0] = [np.zeros_like(r) for r in rhs[0]]      # stops before the first iteration
    rhs[1] = [r * 1e-20 for r in rhs[1]]              # tiny norms: stops on norm_thresh early
    ref = []
    for b, r in zip(hb, rhs):
        h = cmg.Hierarchy(n0, b)
        for l in range(2):
            h.set_rhs(l, r[l])
        o = h.solve(params)
        ref.append((o, [h.phi(l) for l in range(2)]))
        h.close()
    f = cmg.Forest(n0, hb)
    for k in range(3):
        for l in range(2):
            f.set_rhs(k, l, rhs[k][l])
    outs = f.solve(params)
    assert len({o["iterations"] for o, _ in ref}) > 1
    for k, (o, phis) in enumerate(ref):
        assert outs[k]["iterations"] == o["iterations"] and outs[k]["exit_status"] == o["exit_status"], k
        for l in range(2):
            assert np.array_equal(f.phi(k, l), phis[l]), (k, l)
    f.close()
