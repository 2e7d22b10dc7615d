import importlib.util
import json
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_cmg():
    """The ctypes binding of libcmg.so (the package directory name is not an
    importable identifier, so it is loaded by path)."""
    path = os.path.join(ROOT, "chombo_3.2_b200", "cmg.py")
    spec = importlib.util.spec_from_file_location("cmg", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def cmg():
    return load_cmg()


def golden(name):
    meta = json.load(open(os.path.join(GOLDEN, name + ".json")))
    arrays = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    return meta, arrays


def golden_names():
    return sorted(f[:-5] for f in os.listdir(GOLDEN) if f.endswith(".json"))
