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


# Fixtures skipped when CMG_LARGE=0 (the 149M-cell 256^3 workload, about half
# a minute of GPU checks); they run by default.
LARGE = {"config2_vc_3lev_256"}


# Fixtures of the other paths (multilevel BiCGStab, heat solvers, FineInterp),
# which reuse the hierarchies of the AMRMultiGrid fixtures.
OTHER_PATHS = ("bicgstab_", "heat_", "fineinterp_")


def golden_names(include_large=False):
    """The AMRMultiGrid fixtures (host-only checks pass include_large: they
    are quick at every size)."""
    names = sorted(f[:-5] for f in os.listdir(GOLDEN) if f.endswith(".json") and not f.startswith(OTHER_PATHS))
    if not include_large and os.environ.get("CMG_LARGE") == "0":
        names = [n for n in names if n not in LARGE]
    return names


def covered_mask(boxes, finer_boxes):
    """Valid cells of a level (boxes in layout order, x fastest) covered by the
    next finer level (ratio 2): the cells outside the composite solution."""
    if not boxes:
        return np.zeros(0, bool)
    b = np.array(boxes)
    lo, hi = b[:, :3].min(axis=0), b[:, 3:].max(axis=0)
    n = hi - lo + 1
    vol = np.zeros((n[2], n[1], n[0]), bool)
    for f in finer_boxes:
        flo = np.array(f[:3]) // 2 - lo
        fhi = np.array(f[3:]) // 2 - lo
        vol[flo[2]:fhi[2] + 1, flo[1]:fhi[1] + 1, flo[0]:fhi[0] + 1] = True
    masks = []
    for x in boxes:
        a = np.array(x[:3]) - lo
        c = np.array(x[3:]) - lo
        masks.append(vol[a[2]:c[2] + 1, a[1]:c[1] + 1, a[0]:c[0] + 1].ravel())
    return np.concatenate(masks)
