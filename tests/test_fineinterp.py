"""FineInterp without a GPU: the fixtures (recorded from the reference's own
FineInterp.cpp, oracle/_ref/cmg_oracle_fineinterp) against an independent
numpy restatement of interpToFine / pwcinterpToFine (InterpF.ChF:12-369,
FineInterp.cpp:106-399 with the default PCInterp boundary type), the seeded
coarse fields the fixtures use, the oracle reproducing its fixtures, and the
C ABI's argument checks (which run before any device call)."""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden

sys.path.insert(0, GOLDEN)
from make_golden_fineinterp import CASES, seeded_field  # noqa: E402

FIORACLE = os.path.join(ROOT, "oracle", "_ref", "cmg_oracle_fineinterp")


def coarse_input(meta, base):
    """The coarse data of a fixture, or None for the seeded right-hand side."""
    if meta["input"] != "field":
        return None
    lev = meta["level"] - 1
    return seeded_field(base["boxes"][lev], base["n0"] << lev, 1000 + meta["level"])


def fine_interp_numpy(cboxes, coarse, fboxes, nc, pwc):
    """interpToFine restated over a dense copy of the coarse level (n_c^3)."""
    D = np.full((nc, nc, nc), np.nan)  # [i, j, k]
    pos = 0
    for b in cboxes:
        n = (b[3] - b[0] + 1, b[4] - b[1] + 1, b[5] - b[2] + 1)
        blk = coarse[pos:pos + n[0] * n[1] * n[2]].reshape(n[2], n[1], n[0]).transpose(2, 1, 0)
        D[b[0]:b[3] + 1, b[1]:b[4] + 1, b[2]:b[5] + 1] = blk
        pos += blk.size
    out = []
    for fb in fboxes:
        lo = [fb[d] // 2 for d in range(3)]
        hi = [fb[d + 3] // 2 for d in range(3)]
        n = [hi[d] - lo[d] + 1 for d in range(3)]
        sl = tuple(slice(lo[d], hi[d] + 1) for d in range(3))
        v = D[sl]
        f = np.empty((2 * n[0], 2 * n[1], 2 * n[2]))
        for a in range(2):
            for b in range(2):
                for c in range(2):
                    f[a::2, b::2, c::2] = v
        # b_mod = (grow(b, 1) & domain).grow(-1)
        mlo = [max(lo[d] - 1, 0) + 1 for d in range(3)]
        mhi = [min(hi[d] + 1, nc - 1) - 1 for d in range(3)]
        if not pwc and all(mlo[d] <= mhi[d] for d in range(3)):
            ms = tuple(slice(mlo[d], mhi[d] + 1) for d in range(3))
            c0 = D[ms]

            def sh(di, dj, dk):
                return D[mlo[0] + di:mhi[0] + 1 + di, mlo[1] + dj:mhi[1] + 1 + dj, mlo[2] + dk:mhi[2] + 1 + dk]

            s = [0.5 * (sh(1, 0, 0) - sh(-1, 0, 0)), 0.5 * (sh(0, 1, 0) - sh(0, -1, 0)),
                 0.5 * (sh(0, 0, 1) - sh(0, 0, -1))]
            smax, smin = c0.copy(), c0.copy()
            for dk in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    for di in (-1, 0, 1):
                        smax = np.fmax(smax, sh(di, dj, dk))
                        smin = np.fmin(smin, sh(di, dj, dk))
            deltasum = 0.5 * (np.abs(s[0]) + np.abs(s[1]) + np.abs(s[2]))
            eta = np.fmin(smax - c0, c0 - smin)
            tiny = float(np.float32(1.0e-9))
            with np.errstate(divide="ignore", invalid="ignore"):
                eta = np.where(eta <= tiny * np.abs(smax), 0.0, np.where(deltasum > eta, eta / deltasum, 1.0))
            s = [eta * x for x in s]
            o = [2 * (mlo[d] - lo[d]) for d in range(3)]
            m = [mhi[d] - mlo[d] + 1 for d in range(3)]
            for a in range(2):
                for b in range(2):
                    for c in range(2):
                        r = f[o[0] + a:o[0] + 2 * m[0]:2, o[1] + b:o[1] + 2 * m[1]:2, o[2] + c:o[2] + 2 * m[2]:2]
                        r = r + (0.25 if a else -0.25) * s[0]
                        r = r + (0.25 if b else -0.25) * s[1]
                        r = r + (0.25 if c else -0.25) * s[2]
                        f[o[0] + a:o[0] + 2 * m[0]:2, o[1] + b:o[1] + 2 * m[1]:2, o[2] + c:o[2] + 2 * m[2]:2] = r
        out.append(f.transpose(2, 1, 0).ravel())
    return np.concatenate(out)


FIELD_CASES = sorted(n for n, c in CASES.items() if c[3] == "field")


@pytest.mark.parametrize("name", FIELD_CASES)
def test_seeded_field_matches_fixture(name):
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    c = coarse_input(meta, base)
    assert float(np.sum(c)) == meta["coarse_sum"]
    if "coarse" in arrays:
        assert np.array_equal(c, arrays["coarse"])


@pytest.mark.parametrize("name", [n for n in FIELD_CASES if not n.startswith("fineinterp_config1")])
def test_numpy_restatement_matches_reference_fixture(name):
    """The reference's FineInterp output equals the numpy restatement bit for bit."""
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    lev = meta["level"]
    got = fine_interp_numpy(base["boxes"][lev - 1], coarse_input(meta, base), base["boxes"][lev],
                            base["n0"] << (lev - 1), meta["pwc"])
    assert got.size == meta["fine_cells"]
    assert np.array_equal(got[::meta["sample_stride"]], arrays["fine"])


def test_limiter_takes_every_branch():
    """The field fixtures exercise eta = 0, eta = 1 and eta = ratio cells."""
    meta, _ = golden("fineinterp_vc_3lev_16_l2_field")
    base, _ = golden(meta["base"])
    D = np.zeros(3)
    c = coarse_input(meta, base)
    nc = base["n0"] << 1
    dense = np.full((nc, nc, nc), np.nan)
    pos = 0
    for b in base["boxes"][1]:
        n = (b[3] - b[0] + 1, b[4] - b[1] + 1, b[5] - b[2] + 1)
        dense[b[0]:b[3] + 1, b[1]:b[4] + 1, b[2]:b[5] + 1] = c[pos:pos + n[0] * n[1] * n[2]].reshape(
            n[2], n[1], n[0]).transpose(2, 1, 0)
        pos += n[0] * n[1] * n[2]
    inner = dense[1:-1, 1:-1, 1:-1]
    ok = ~np.isnan(inner)
    for dk in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                ok &= ~np.isnan(dense[1 + di:nc - 1 + di, 1 + dj:nc - 1 + dj, 1 + dk:nc - 1 + dk])
    s = [0.5 * (dense[2:, 1:-1, 1:-1] - dense[:-2, 1:-1, 1:-1]), 0.5 * (dense[1:-1, 2:, 1:-1] - dense[1:-1, :-2, 1:-1]),
         0.5 * (dense[1:-1, 1:-1, 2:] - dense[1:-1, 1:-1, :-2])]
    smax, smin = inner.copy(), inner.copy()
    for dk in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                w = dense[1 + di:nc - 1 + di, 1 + dj:nc - 1 + dj, 1 + dk:nc - 1 + dk]
                smax, smin = np.fmax(smax, w), np.fmin(smin, w)
    deltasum = 0.5 * (np.abs(s[0]) + np.abs(s[1]) + np.abs(s[2]))
    eta = np.fmin(smax - inner, inner - smin)[ok]
    deltasum = deltasum[ok]
    zero = eta <= float(np.float32(1e-9)) * np.abs(smax[ok])
    D[0] = np.count_nonzero(zero)
    D[1] = np.count_nonzero(~zero & (deltasum > eta))
    D[2] = np.count_nonzero(~zero & (deltasum <= eta))
    assert np.all(D > 0), D


@pytest.mark.skipif(not os.path.exists(FIORACLE), reason="oracle not built (needs the reference tree)")
@pytest.mark.parametrize("name", [n for n in sorted(CASES) if not n.startswith("fineinterp_config1")])
def test_fineinterp_oracle_reproduces_golden(tmp_path, name):
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    out = str(tmp_path / name)
    cmd = [FIORACLE] + base["args"].split() + [f"level={meta['level']}", f"pwc={meta['pwc']}", "out=" + out]
    c = coarse_input(meta, base)
    if c is not None:
        c.tofile(out + ".coarse")
        cmd.append("coarse=" + out + ".coarse")
    subprocess.run(cmd, check=True, capture_output=True, timeout=300)
    got = json.load(open(out + ".json"))
    assert got["fine_boxes"] == base["boxes"][meta["level"]]
    raw = np.fromfile(out + ".bin", dtype=np.float64)
    assert np.array_equal(raw[::meta["sample_stride"]], arrays["fine"])


def test_fine_interp_create_rejects_bad_layouts(cmg):
    L = cmg.lib()
    h = ctypes.c_void_p()
    dom_lo, dom_hi = (ctypes.c_int * 3)(0, 0, 0), (ctypes.c_int * 3)(31, 31, 31)
    coarse = cmg.boxes_array([(0, 0, 0, 15, 15, 15)])
    # a fine box not coarsenable by 2
    rc = L.cmg_fine_interp_create(dom_lo, dom_hi, 1, cmg.boxes_array([(1, 0, 0, 8, 7, 7)]), 1, coarse,
                                  ctypes.byref(h))
    assert rc == cmg.CMG_EINVAL and "coarsenable" in L.cmg_last_error().decode()
    # a fine box outside the fine domain
    rc = L.cmg_fine_interp_create(dom_lo, dom_hi, 1, cmg.boxes_array([(24, 24, 24, 33, 31, 31)]), 1, coarse,
                                  ctypes.byref(h))
    assert rc == cmg.CMG_EINVAL
    # a coarse box outside the coarse domain
    rc = L.cmg_fine_interp_create(dom_lo, dom_hi, 1, cmg.boxes_array([(0, 0, 0, 7, 7, 7)]), 1,
                                  cmg.boxes_array([(0, 0, 0, 16, 15, 15)]), ctypes.byref(h))
    assert rc == cmg.CMG_EINVAL
    assert L.cmg_interp_to_fine(None, 1, 0) == cmg.CMG_EINVAL
