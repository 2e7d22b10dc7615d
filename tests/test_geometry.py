"""Host geometry against the reference: base-level splitting and the Copier
motion plans (exchange and coarsened-fine -> coarse) must match bit for bit,
item for item, in order."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, golden_names

CASES = golden_names(include_large=True)


@pytest.mark.parametrize("name", CASES)
def test_domain_split_matches_reference(cmg, name):
    meta, _ = golden(name)
    n0, maxbox, block = meta["n0"], meta["maxbox"], meta["block"]
    boxes = cmg.domain_split((0, 0, 0), (n0 - 1,) * 3, maxbox, block)
    assert [list(b) for b in boxes] == meta["boxes"][0]


def plan_arrays(name):
    """The complete reference plans of the benchmark-size fixtures, whose JSON
    keeps only the plan sizes (tests/golden/make_golden_plans.py)."""
    path = os.path.join(GOLDEN, name + "_plans.npz")
    return dict(np.load(path)) if os.path.exists(path) else None


def as_items(plan):
    return [[int(r[0]), int(r[1]), list(map(int, r[2:8])), list(map(int, r[8:14]))] for r in plan]


def ref_items(plan):
    return [[m[0], m[1], m[2], m[3]] for m in plan]


@pytest.mark.parametrize("name", CASES)
def test_exchange_plans_match_reference(cmg, name):
    meta, _ = golden(name)
    bc = meta.get("bc", "")
    periodic = [len(bc) == 6 and bc[2 * d] == "P" for d in range(3)]
    for lev, boxes in enumerate(meta["boxes"]):
        if any(periodic):
            n = meta["n0"] << lev
            plan = cmg.layout_exchange_plan_periodic(boxes, (0, 0, 0, n - 1, n - 1, n - 1), periodic)
        else:
            plan = cmg.layout_exchange_plan(boxes)
        if "exchange_plans" in meta:
            assert as_items(plan) == ref_items(meta["exchange_plans"][lev]), f"level {lev}"
        else:
            ref = plan_arrays(name)[f"exchange{lev}"]
            assert len(plan) == meta["exchange_plan_sizes"][lev] == len(ref)
            assert np.array_equal(np.asarray(plan, dtype=np.int64), ref.astype(np.int64)), f"level {lev}"


@pytest.mark.parametrize("name", CASES)
def test_coarse_fine_plans_match_reference(cmg, name):
    meta, _ = golden(name)
    for lev in range(1, len(meta["boxes"])):
        plan = cmg.layout_coarse_fine_plan(meta["boxes"][lev], meta["boxes"][lev - 1])
        if "coarsened_fine_plans" in meta:
            assert as_items(plan) == ref_items(meta["coarsened_fine_plans"][lev - 1]), f"level {lev}"
        else:
            ref = plan_arrays(name)[f"coarsened_fine{lev}"]
            assert len(plan) == meta["coarsened_fine_plan_sizes"][lev - 1] == len(ref)
            assert np.array_equal(np.asarray(plan, dtype=np.int64), ref.astype(np.int64)), f"level {lev}"


def test_fine_levels_nest_in_coarse(cmg):
    for name in CASES:
        meta, _ = golden(name)
        for lev in range(1, len(meta["boxes"])):
            plan = cmg.layout_coarse_fine_plan(meta["boxes"][lev], meta["boxes"][lev - 1])
            covered = sum(int(np.prod(np.array(r[11:14]) - np.array(r[8:11]) + 1)) for r in plan)
            fine = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in meta["boxes"][lev])
            assert covered * 8 == fine, (name, lev)
