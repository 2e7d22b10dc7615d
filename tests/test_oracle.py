"""The oracle (test infrastructure): the reference's own AMRMultiGrid solve
compiled from its C++ sources with a C++ restatement of its ChF kernels
(oracle/Makefile).  These CPU tests pin it:

* it reproduces the committed golden fixtures bit for bit (box layouts from
  domainSplit/BRMeshRefine, residual history, exit status, phi), so the
  fixtures the GPU parity tests use are the reference's own output;
* the reference's own AMRTools tests (lib/test/AMRTools), built against the
  restated kernels, pass: quadCFInterpTest (QUADINTERP, PHISTAR and the
  QuadCFStencil derivatives, relative error <= 1e-12 on quadratics) and
  testCoarseAverage (AVERAGE).  fluxRegisterTest is listed in the
  reference's own skip list (lib/test/AMRTools/skip_these.txt) and fails
  there too, so it is recorded, not asserted.

Both need the oracle built from the reference tree (make -C oracle all
reftests); they skip where it was not built."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden

ORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle")
REFTESTS = os.path.join(ROOT, "oracle", "_ref", "tests")

needs_oracle = pytest.mark.skipif(not os.path.exists(ORACLE), reason="oracle not built (needs the reference tree)")


@needs_oracle
@pytest.mark.parametrize("name", ["poisson_1lev_32", "helmholtz_1lev_32", "vc_1lev_32", "poisson_3lev_16",
                                  "helmholtz_2lev_16", "vc_3lev_16", "poisson_3lev_16_walls", "vc_3lev_16_walls",
                                  "helmholtz_1lev_32_periodic", "helmholtz_1lev_32_ppnndd", "vc_1lev_32_periodic"])
def test_oracle_reproduces_golden(tmp_path, name):
    meta, arrays = golden(name)
    out = str(tmp_path / name)
    subprocess.run([ORACLE] + meta["args"].split() + ["out=" + out], check=True, capture_output=True, timeout=300)
    got = json.load(open(out + ".json"))
    assert got["boxes"] == meta["boxes"]
    assert got["exit_status"] == meta["exit_status"]
    assert got["residual_history"] == meta["residual_history"]
    raw = np.fromfile(out + ".bin", dtype=np.float64)
    pos = 0
    for lev, boxes in enumerate(meta["boxes"]):
        n = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in boxes)
        rhs, phi = raw[pos:pos + n], raw[pos + n:pos + 2 * n]
        pos += 2 * n
        if meta["op"] == 1:
            pos += n + sum((b[3] - b[0] + 1 + (d == 0)) * (b[4] - b[1] + 1 + (d == 1)) * (b[5] - b[2] + 1 + (d == 2))
                           for d in range(3) for b in boxes)
        assert np.array_equal(phi, arrays[f"phi{lev}"])
        assert float(np.sum(rhs)) == meta["rhs_sum"][lev]


@pytest.mark.parametrize("test", ["quadCFInterpTest", "testCoarseAverage", "testFineInterp"])
def test_reference_amrtools_test_passes(test):
    exe = os.path.join(REFTESTS, test)
    if not os.path.exists(exe):
        pytest.skip("reference tests not built (make -C oracle reftests)")
    r = subprocess.run([exe], capture_output=True, timeout=600, cwd=REFTESTS)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


MLORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_mlbicgstab")


@pytest.mark.skipif(not os.path.exists(MLORACLE), reason="oracle not built (needs the reference tree)")
@pytest.mark.parametrize("name", ["bicgstab_poisson_1lev_32", "bicgstab_vc_3lev_16"])
def test_bicgstab_oracle_reproduces_golden(tmp_path, name):
    """The reference's BiCGStab over MultilevelLinearOp reproduces its fixture bit for bit."""
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    out = str(tmp_path / name)
    subprocess.run([MLORACLE] + base["args"].split() + meta["solver_args"].split() + ["out=" + out], check=True,
                   capture_output=True, timeout=300)
    got = json.load(open(out + ".json"))
    for k in ("exit_status", "iterations", "initial_residual", "final_residual"):
        assert got[k] == meta[k], k
    raw = np.fromfile(out + ".bin", dtype=np.float64)
    pos = 0
    for lev, boxes in enumerate(base["boxes"]):
        n = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in boxes)
        assert np.array_equal(raw[pos:pos + n][::meta["sample_stride"]], arrays[f"phi{lev}"])
        pos += n


HEATORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_heat")


@pytest.mark.skipif(not os.path.exists(HEATORACLE), reason="oracle not built (needs the reference tree)")
@pytest.mark.parametrize("name", ["heat_poisson_1lev_32", "heat_vc_3lev_16", "heat_tga_vc_3lev_16"])
def test_heat_oracle_reproduces_golden(tmp_path, name):
    """The reference's BackwardEuler steps reproduce their fixture bit for bit."""
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    out = str(tmp_path / name)
    grid = [a for a in base["args"].split() if a.split("=")[0] not in ("op", "alpha", "beta")]
    subprocess.run([HEATORACLE] + grid + meta["heat_args"].split() + ["out=" + out], check=True,
                   capture_output=True, timeout=300)
    got = json.load(open(out + ".json"))
    assert got["exit_status"] == meta["exit_status"] and got["iterations"] == meta["iterations"]
    raw = np.fromfile(out + ".bin", dtype=np.float64)
    pos = 0
    for lev, boxes in enumerate(base["boxes"]):
        n = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in boxes)
        assert np.array_equal(raw[pos:pos + n], arrays[f"phi{lev}"])
        pos += n
