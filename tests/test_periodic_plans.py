"""Exchange plans on periodic domains against the reference's own Copier, run here through the oracle build
(oracle/_ref/cmg_oracle plansonly=1): corner cases beside the golden fixtures -- a single box that is its own
periodic neighbour in every direction, two boxes along one periodic direction, and directions periodic in
some axes only.  Items and their order must be the same."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle")

CASES = [
    ("n0=16 levels=1 maxbox=16 block=8 op=0 alpha=1 beta=-0.1 bc=PPPPPP", 16, 16),
    ("n0=16 levels=1 maxbox=8 block=8 op=0 alpha=1 beta=-0.1 bc=PPPPPP", 16, 8),
    ("n0=32 levels=1 maxbox=16 block=8 op=0 alpha=1 beta=-0.1 bc=PPDDNN", 32, 16),
    ("n0=32 levels=1 maxbox=8 block=8 op=1 alpha=1 beta=-1 bc=NDPPPP", 32, 8),
]


def reference_plan(args, tmp):
    out = str(tmp / "plans")
    subprocess.run([ORACLE] + args.split() + ["plansonly=1", "out=" + out], check=True, capture_output=True,
                   timeout=120)
    raw = np.fromfile(out + ".plans", dtype=np.int32)
    n = int(raw[0])
    return raw[1:1 + 14 * n].reshape(n, 14)


@pytest.mark.skipif(not os.path.exists(ORACLE), reason="oracle not built (needs the reference tree)")
@pytest.mark.parametrize("args,n0,maxbox", CASES)
def test_periodic_exchange_plan_matches_reference(cmg, tmp_path, args, n0, maxbox):
    bc = args.split("bc=")[1].split()[0]
    periodic = [bc[2 * d] == "P" for d in range(3)]
    boxes = cmg.domain_split((0, 0, 0), (n0 - 1,) * 3, maxbox, 8)
    ours = cmg.layout_exchange_plan_periodic(boxes, (0, 0, 0, n0 - 1, n0 - 1, n0 - 1), periodic)
    ref = reference_plan(args, tmp_path)
    assert ours.shape == ref.shape, (ours.shape, ref.shape)
    assert np.array_equal(np.asarray(ours, dtype=np.int64), ref.astype(np.int64))
