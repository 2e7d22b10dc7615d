"""The GPU operator factories accept only the homogeneous Dirichlet boundary
condition the device solve applies: define() probes the BCHolder on the six
domain faces and stops with MayDay::Error on anything else.  A Chombo program
(oracle/dropin.cpp, built against the reference's objects) hands a Neumann
condition to cmg_chombo::GpuAMRPoissonOpFactory::define; no device is
touched before the refusal."""
import os
import subprocess

import pytest

from conftest import ROOT

DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")


def test_neumann_boundary_condition_is_refused():
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN, "n0=16", "levels=2", "maxbox=8", "block=4", "op=0", "alpha=0", "beta=1",
                        "neumann=1"], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0, r.stdout
    assert "neumann_accepted" not in r.stdout
    assert "homogeneous Dirichlet boundary conditions only" in (r.stdout + r.stderr)
