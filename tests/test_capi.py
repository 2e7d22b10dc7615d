"""C-ABI library: loads, exports every entry point of include/cmg.h, and
rejects bad arguments with status codes (no device needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cmg.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(cmg_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(cmg):
    lib = cmg.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_domain_split_rejects_bad_arguments(cmg):
    lib = cmg.lib()
    n = ctypes.c_int()
    lo, hi = (ctypes.c_int * 3)(0, 0, 0), (ctypes.c_int * 3)(62, 63, 63)  # 63 cells: not coarsenable by 8
    rc = lib.cmg_domain_split(lo, hi, 32, 8, None, 0, ctypes.byref(n))
    assert rc == cmg.CMG_EINVAL
    assert b"coarsenable" in lib.cmg_last_error()


def test_hierarchy_create_rejects_overlapping_boxes(cmg):
    with pytest.raises(cmg.CmgError) as e:
        cmg.Hierarchy(16, [[(0, 0, 0, 9, 15, 15), (8, 0, 0, 15, 15, 15)]])
    assert e.value.code == cmg.CMG_EINVAL


def test_hierarchy_create_rejects_box_outside_domain(cmg):
    with pytest.raises(cmg.CmgError) as e:
        cmg.Hierarchy(16, [[(0, 0, 0, 16, 15, 15)]])
    assert e.value.code == cmg.CMG_EINVAL


def test_null_hierarchy_is_an_error(cmg):
    lib = cmg.lib()
    out = ctypes.c_int64()
    assert lib.cmg_num_cells(None, 0, ctypes.byref(out)) == cmg.CMG_EINVAL


def test_hierarchy_create_rejects_half_periodic_direction(cmg):
    with pytest.raises(cmg.CmgError) as e:
        cmg.Hierarchy(16, [[(0, 0, 0, 15, 15, 15)]], bc="PDNNDD")
    assert e.value.code == cmg.CMG_EINVAL


def test_hierarchy_create_rejects_periodic_amr(cmg):
    # periodic directions on one-level hierarchies only; refused before any device work
    with pytest.raises(cmg.CmgError) as e:
        cmg.Hierarchy(16, [[(0, 0, 0, 15, 15, 15)], [(8, 8, 8, 15, 15, 15)]], bc="PPPPPP")
    assert e.value.code == cmg.CMG_EINVAL
    assert "one-level" in str(e.value)
