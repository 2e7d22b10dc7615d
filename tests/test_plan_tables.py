"""Regression check of the host plan builders: a field-wise hash of every plan table (ghost lists, face rules,
per-chunk ghosts, coarse-fine stencils, flux registers, coarse-fine copy items, chunks) of three synthetic
hierarchies (32^3, 64^3 and 128^3 bases, three levels) and of a periodic 64^3 level with its multigrid depths and
bottom plan must stay what it was when the device solve was last
verified against the reference with these tables.  Speed-ups of the builders (threads, indexes, allocation) must
leave these hashes unchanged; a change of the tables themselves needs the GPU parity suite and a new hash."""
import os
import subprocess

from conftest import ROOT

SRC = os.path.join(ROOT, "chombo_3.2_b200", "csrc")
EXPECTED = {32: "3432525cfc94064c", 64: "c526961acb710626", 128: "3a54d17b089c9568"}


def test_plan_tables_unchanged(tmp_path):
    exe = str(tmp_path / "plan_hash")
    srcs = [os.path.join(ROOT, "tests", "cpp", "plan_hash.cpp")] + [os.path.join(SRC, f) for f in
                                                                    ("plan.cpp", "geom.cpp", "meshrefine.cpp",
                                                                     "hostpool.cpp", "hostmem.cpp")]
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", SRC, "-I", "/usr/local/cuda/include",
                        "-o", exe] + srcs + ["-lpthread"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    got = {int(line.split()[1]): line.split()[5] for line in out.stdout.splitlines() if line.startswith("n0 ")}
    assert got == EXPECTED, got
    periodic = [line.split()[-1] for line in out.stdout.splitlines() if line.startswith("periodic64")]
    assert periodic == ["d4c2228b1e0c650f"], periodic
