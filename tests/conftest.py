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


# Fixtures whose GPU checks take minutes (the 149M-cell 256^3 workload); run
# them with CMG_LARGE=1.
LARGE = {"config2_vc_3lev_256"}


# Fixtures of the other paths (multilevel BiCGStab, heat solvers, FineInterp),
# which reuse the hierarchies of the AMRMultiGrid fixtures.
OTHER_PATHS = ("bicgstab_", "heat_", "fineinterp_")


def golden_names():
    """The AMRMultiGrid fixtures."""
    names = sorted(f[:-5] for f in os.listdir(GOLDEN) if f.endswith(".json") and not f.startswith(OTHER_PATHS))
    if os.environ.get("CMG_LARGE") != "1":
        names = [n for n in names if n not in LARGE]
    return names


def covered_mask(boxes, finer_boxes):
    """Valid cells of a level (boxes in layout order, x fastest) covered by the
    next finer level (ratio 2): the cells outside the composite solution."""
    masks = []
    fine = [(np.array(b[:3]) // 2, np.array(b[3:]) // 2) for b in finer_boxes]
    for b in boxes:
        lo, hi = np.array(b[:3]), np.array(b[3:])
        n = hi - lo + 1
        m = np.zeros((n[2], n[1], n[0]), bool)
        for flo, fhi in fine:
            a, c = np.maximum(lo, flo), np.minimum(hi, fhi)
            if np.all(a <= c):
                m[a[2] - lo[2]:c[2] - lo[2] + 1, a[1] - lo[1]:c[1] - lo[1] + 1, a[0] - lo[0]:c[0] - lo[0] + 1] = True
        masks.append(m.ravel())
    return np.concatenate(masks) if masks else np.zeros(0, bool)
