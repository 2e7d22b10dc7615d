"""The GPU operator factories accept the boundary conditions the device solve
applies, homogeneous Dirichlet or homogeneous Neumann on each domain face:
define() probes the BCHolder on the six domain faces, records each face's
type, and stops with MayDay::Error on anything else.  A Chombo program
(oracle/dropin.cpp, built against the reference's objects) hands the
problem's BC function (Dirichlet or Neumann per face, as the AMRINS
projection's pressure BC sets them) and an inhomogeneous Dirichlet one to
cmg_chombo::GpuAMRPoissonOpFactory::define; no device is touched."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")
BASE = ["n0=16", "levels=2", "maxbox=8", "block=4", "op=0", "alpha=0", "beta=1"]


def need_dropin():
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")


def test_inhomogeneous_boundary_condition_is_refused():
    need_dropin()
    r = subprocess.run([DROPIN] + BASE + ["badbc=1"], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0, r.stdout
    assert "inhomogeneous_accepted" not in r.stdout
    assert "homogeneous Neumann (ghost = inside) boundary conditions only" in (r.stdout + r.stderr)


@pytest.mark.parametrize("faces", ["DDDDDD", "NNNNND", "NDNDNN", "NNNNNN", "PPPPPP", "PPNNDD", "DNPPNN"])
def test_face_types_are_read_off_the_bc_function(faces):
    """Periodic directions come from the ProblemDomain (the BC function is not called across them)."""
    need_dropin()
    r = subprocess.run([DROPIN] + BASE + ["bcprobe=1", "bc=" + faces], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["bc_types"] == [{"D": 0, "N": 1, "P": 2}[c] for c in faces]
