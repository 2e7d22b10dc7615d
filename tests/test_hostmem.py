"""The kept large host blocks behind the plan tables (chombo_3.2_b200/csrc/hostmem.*),
compiled with a small C++ driver, and the C ABI's cmg_host_blocks through the library
(host only, no GPU needed)."""
import os
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "chombo_3.2_b200", "csrc")


def test_hostmem(tmp_path):
    exe = str(tmp_path / "hostmem_check")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-I", SRC, "-o", exe,
                        os.path.join(ROOT, "tests", "cpp", "hostmem_check.cpp"), os.path.join(SRC, "hostmem.cpp"),
                        "-lpthread"], capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        pytest.fail(r.stderr[-2000:])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert "hostmem ok" in out.stdout


def test_host_blocks_abi(cmg):
    assert cmg.host_blocks(release=True) == 0
    assert cmg.host_blocks() == 0
