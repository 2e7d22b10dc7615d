"""The host thread pool behind the plan builders, grid generation and host
fills (chombo_3.2_b200/csrc/hostpool.*), compiled with a small C++ driver:
every item once, nested concurrent calls finish, exceptions reach the caller."""
import os
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "chombo_3.2_b200", "csrc")


def test_hostpool(tmp_path):
    exe = str(tmp_path / "hostpool_check")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-I", SRC, "-o", exe,
                        os.path.join(ROOT, "tests", "cpp", "hostpool_check.cpp"), os.path.join(SRC, "hostpool.cpp"),
                        "-lpthread"], capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        pytest.fail(r.stderr[-2000:])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert "hostpool ok" in out.stdout
