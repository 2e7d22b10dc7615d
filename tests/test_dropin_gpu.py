"""The Chombo-side drop-in (include/cmg_chombo.H): a Chombo program built
against the reference's own headers and objects (oracle/dropin.cpp) solves
one seeded hierarchy through the reference's AMRMultiGrid on the CPU and
through cmg_chombo::GpuAMRMultiGrid with the same define / setSolverParameters
/ solve calls.  Exit status and iteration count must be identical, every
residual-history entry within 1e-12 of the initial residual, and phi within
1e-12 relative L-infinity on every level."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")
TOL = 1e-12

CASES = {
    "vc_3lev_16": "n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=-1",
    "poisson_3lev_16": "n0=16 levels=3 maxbox=8 block=4 op=0 alpha=0 beta=1",
    "helmholtz_2lev_16": "n0=16 levels=2 maxbox=8 block=4 op=0 alpha=1 beta=-1",
    "vc_1lev_32": "n0=32 levels=1 maxbox=16 op=1 alpha=1 beta=-1",
    # the AMRINS projection's solves (CCProjector::defineMultiGrid, CCProjector.cpp:1872-1957): a composite
    # Poisson problem with AMRPoissonOpFactory, Neumann walls and a Dirichlet outflow face, a RelaxSolver bottom
    # and m_eps 1e-10
    "projection_3lev_32": "n0=32 levels=3 maxbox=16 block=4 op=0 alpha=0 beta=1 bc=NNNNND relaxbottom=1 eps=1e-10",
    "projection_2lev_16_relax": "n0=16 levels=2 maxbox=8 block=4 op=0 alpha=0 beta=1 bc=NDNNNN relaxbottom=1",
    "vc_3lev_16_walls": "n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=-1 bc=NDNDNN",
    # one-level periodic domains (ProblemDomain periodic in every direction, or in x and y)
    "helmholtz_1lev_32_periodic": "n0=32 levels=1 maxbox=16 op=0 alpha=1 beta=-0.1 bc=PPPPPP",
    "vc_1lev_32_ppnndd": "n0=32 levels=1 maxbox=16 op=1 alpha=1 beta=-1 bc=PPNNDD",
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_matches_reference_solver(name):
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN] + CASES[name].split(), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["gpu_exit"] == out["cpu_exit"], out
    assert out["gpu_iters"] == out["cpu_iters"], out
    assert out["same_history_length"], out
    assert out["history_dev"] <= TOL, out
    assert out["phi_rel_dev"] <= TOL, out
    # bit for bit
    assert out["history_dev"] == 0.0 and out["phi_rel_dev"] == 0.0, out
    # computeAMRResidual through the drop-in reproduces the solve's last entry.
    assert out["gpu_final_residual"] == out["gpu_history_last"], out


BICG_CASES = {
    "vc_3lev_16": "n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=-1 bicgstab=1 mgiters=2 mgsmooth=4 eps=1e-9",
    "poisson_1lev_32": "n0=32 levels=1 maxbox=16 op=0 alpha=0 beta=1 bicgstab=1 mgiters=1 mgsmooth=4 eps=1e-9",
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(BICG_CASES))
def test_dropin_bicgstab_matches_reference_solver(name):
    """MultilevelLinearOp + BiCGStabSolver<Vector<LevelData*>> (the variable-coefficient example's solve path)
    against cmg_chombo::GpuMultilevelLinearOp + GpuMultilevelBiCGStabSolver with the same calls."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN] + BICG_CASES[name].split(), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["gpu_exit"] == out["cpu_exit"] == 1, out
    assert out["gpu_iters"] == out["cpu_iters"], out
    assert abs(out["gpu_r0"] - out["cpu_r0"]) <= TOL * out["cpu_r0"], out
    assert abs(out["gpu_rfinal"] - out["cpu_rfinal"]) <= TOL * out["cpu_r0"], out
    assert out["phi_rel_dev"] <= TOL, out


HEAT_CASES = {
    "euler_poisson_3lev_16": "n0=16 levels=3 maxbox=8 block=4 op=0 alpha=1 beta=1 heat=1 dt=1e-3 steps=2",
    "tga_vc_3lev_16": "n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=1 heat=2 dt=1e-6 steps=2",
    "tga_poisson_1lev_32": "n0=32 levels=1 maxbox=16 op=0 alpha=1 beta=1 heat=2 dt=1e-3 steps=2",
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(HEAT_CASES))
def test_dropin_heat_matches_reference_solver(name):
    """BackwardEuler / AMRTGA over AMRMultiGrid against cmg_chombo::GpuBackwardEuler / GpuAMRTGA over
    GpuAMRMultiGrid with the same calls."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN] + HEAT_CASES[name].split(), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["gpu_exit"] == out["cpu_exit"] == 1, out
    assert out["phi_rel_dev"] <= TOL, out


FINEINTERP_CASES = {
    "fineinterp_vc_3lev_16": "n0=16 levels=3 maxbox=8 block=4 fineinterp=1",
    "fineinterp_poisson_3lev_32": "n0=32 levels=3 maxbox=16 fineinterp=1",
    "fineinterp_pwc_poisson_3lev_32": "n0=32 levels=3 maxbox=16 fineinterp=2",
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FINEINTERP_CASES))
def test_dropin_fineinterp_matches_reference(name):
    """FineInterp against cmg_chombo::GpuFineInterp with the same calls: bit for bit."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN] + FINEINTERP_CASES[name].split(), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["cells"] > 0 and out["max_abs_diff"] == 0.0, out


OPS_CASES = {
    "vc_3lev_16": "n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=-1",
    "poisson_3lev_32": "n0=32 levels=3 maxbox=16 block=4 op=0 alpha=0 beta=1",
    "helmholtz_2lev_16": "n0=16 levels=2 maxbox=8 block=4 op=0 alpha=1 beta=-1",
    # Neumann walls with a Dirichlet outflow face (the AMRINS projection's pressure BC) and mixed faces
    "poisson_3lev_32_walls": "n0=32 levels=3 maxbox=16 block=4 op=0 alpha=0 beta=1 bc=NNNNND",
    "vc_3lev_16_walls": "n0=16 levels=3 maxbox=8 block=4 op=1 alpha=1 beta=-1 bc=NDNDNN",
    "projection_3lev_32": "n0=32 levels=3 maxbox=16 block=4 op=0 alpha=0 beta=1 bc=NNNNND relaxbottom=1",
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(OPS_CASES))
def test_each_operator_matches_reference_bit_for_bit(name):
    """The reference's AMRPoissonOp / VCAMRPoissonOp2 and the GPU AMRLevelOps (cmg_chombo::GpuAMRPoissonOp) get
    the same LevelData inputs, one method at a time: residual, applyOp, relax, preCond, the AMROperator /
    AMRResidual family with coarse-fine interpolation and reflux, AMRRestrictS, assignCopier, zeroCovered,
    AMRProlongS, AMRUpdateResidual, QuadCFInterp::coarseFineInterp (ghost cells), norms, dot products, BLAS-1,
    and on every multigrid depth residual, relax, preCond, restrictResidual, prolongIncrement.  Every valid cell
    of every output is equal (the operator family on levels with a finer level compares the cells not under it:
    the reference's flux register also writes covered cells, which every caller discards)."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN] + OPS_CASES[name].split() + ["ops=1"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    ops = out["ops"]
    names = {o["op"] for o in ops}
    for needed in ("residual", "applyOp", "relax2", "preCond", "AMROperator", "AMRResidual", "AMRRestrictS",
                   "assignCopier", "AMRProlongS", "AMRUpdateResidual", "coarseFineInterp", "restrictResidual",
                   "prolongIncrement", "norm2", "dotProduct", "axby"):
        assert needed in names, (needed, sorted(names))
    bad = [o for o in ops if o["ndiff"] != 0]
    assert not bad, bad
    assert all(o["cells"] > 0 for o in ops), ops


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(OPS_CASES))
def test_reference_amrmultigrid_over_gpu_operators(name):
    """The reference's own AMRMultiGrid, unmodified, defined once with the reference factory and once with the
    GPU factory (an AMRLevelOpFactory<LevelData<FArrayBox>>): identical exit status, iteration count, residual
    history and phi, bit for bit."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN] + OPS_CASES[name].split() + ["amrmg=1"], capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["gpu_exit"] == out["cpu_exit"] == 1, out
    assert out["gpu_iters"] == out["cpu_iters"], out
    assert out["history_exact"], out
    assert out["phi_ndiff"] == 0, out


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(OPS_CASES))
def test_reference_amrfasmultigrid_over_gpu_operators(name):
    """The reference's AMRFASMultiGrid (V-cycle mode, AMRFASMultiGrid.H), unmodified, over the reference factory
    and over the GPU factory: it drives the operators through relaxNF, AMRRestrictS with and without the
    residual, AMROperatorNC on the coarse level's own coarse-fine ghosts, AMRProlongS and the FASMultiGrid
    depths below level 0.  Same exit status, iteration count, final composite residual and phi, bit for bit."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in check not built (make -C oracle dropin, needs the reference tree)")
    r = subprocess.run([DROPIN] + OPS_CASES[name].split() + ["amrmg=1", "fas=1", "iters=12"], capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["fas"] == 1
    assert out["gpu_exit"] == out["cpu_exit"], out
    assert out["gpu_iters"] == out["cpu_iters"] > 0, out
    assert out["history_exact"], out
    assert out["phi_ndiff"] == 0, out
