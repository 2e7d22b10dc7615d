"""The reference arm of bench.py on the periodic configuration (the reference's OpenMP solve on the host cores,
capped at 2 V-cycles): runs without a GPU and prints the contract's JSON line."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

OMPORACLE = os.path.join(ROOT, "oracle", "_ref", "omp", "cmg_oracle")


@pytest.mark.skipif(not os.path.exists(OMPORACLE), reason="OpenMP oracle not built (needs the reference tree)")
def test_periodic_reference_arm_prints_its_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "periodic", "--impl",
                        "reference", "--n0", "64"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "solves/s"
    assert line["s_per_vcycle"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0
