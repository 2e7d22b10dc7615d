"""FineInterp on the device (cmg_interp_to_fine on a hierarchy's phi, and the
standalone cmg_fine_interp object) against the reference's FineInterp output
recorded in the fixtures: bit for bit.  At the config-1 sizes, properties
that hold exactly: a constant stays constant, scaling the coarse data by a
power of two scales the fine data by it, and piecewise-constant
interpolation copies every parent."""
import numpy as np
import pytest

from conftest import golden
from test_fineinterp import CASES, coarse_input


def setup(cmg, name):
    meta, arrays = golden(name)
    base, _ = golden(meta["base"])
    h = cmg.Hierarchy(base["n0"], base["boxes"], op=base["op"], alpha=base["alpha"], beta=base["beta"], bc=base.get("bc"))
    lev = meta["level"]
    c = coarse_input(meta, base)
    if c is None:
        h.fill_synthetic(base["seed"])
        c = h.get_rhs(lev - 1)
    return meta, arrays, base, h, c


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_interp_to_fine_matches_reference(cmg, name):
    meta, arrays, base, h, c = setup(cmg, name)
    lev = meta["level"]
    h.set_phi(lev - 1, c)
    h.set_phi(lev, np.full(h.num_cells(lev), 7.0))
    h.interp_to_fine(lev, pwc=bool(meta["pwc"]))
    got = h.phi(lev)
    assert got.size == meta["fine_cells"]
    assert np.array_equal(got[::meta["sample_stride"]], arrays["fine"])
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_standalone_fine_interp_matches_reference(cmg, name):
    meta, arrays, base, h, c = setup(cmg, name)
    h.close()
    lev = meta["level"]
    nf = base["n0"] << lev
    fi = cmg.FineInterp((0, 0, 0, nf - 1, nf - 1, nf - 1), base["boxes"][lev], base["boxes"][lev - 1])
    got = fi.interp_to_fine(c, pwc=bool(meta["pwc"]))
    assert np.array_equal(got[::meta["sample_stride"]], arrays["fine"])
    fi.close()


@pytest.mark.gpu
def test_exact_properties_at_config1_size(cmg):
    meta, arrays, base, h, c = setup(cmg, "fineinterp_config1_vc_3lev_128_l2")
    h.set_phi(1, c)
    h.interp_to_fine(2)
    ref = h.phi(2)
    h.set_phi(1, 4.0 * c)
    h.interp_to_fine(2)
    assert np.array_equal(h.phi(2), 4.0 * ref)
    h.set_phi(1, np.full(c.size, -0.375))
    h.interp_to_fine(2)
    assert np.all(h.phi(2) == -0.375)
    # piecewise constant: every fine cell holds its parent's value
    h.set_phi(1, c)
    h.interp_to_fine(2, pwc=True)
    pwc = h.phi(2)
    cb, fbox = base["boxes"][1], base["boxes"][2]
    parent = {}
    pos = 0
    for b in cb:
        n = (b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1)
        parent[tuple(b)] = (pos, b)
        pos += n
    # check one fine box per 50 against its coarse parent cells
    fpos = 0
    for t, b in enumerate(fbox):
        n = (b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1)
        if t % 50 == 0:
            k, j, i = np.meshgrid(np.arange(b[2], b[5] + 1), np.arange(b[1], b[4] + 1), np.arange(b[0], b[3] + 1),
                                  indexing="ij")
            I, J, K = i.ravel() // 2, j.ravel() // 2, k.ravel() // 2
            want = np.empty(n)
            for p0, q in parent.values():
                m = (I >= q[0]) & (I <= q[3]) & (J >= q[1]) & (J <= q[4]) & (K >= q[2]) & (K <= q[5])
                nx, ny = q[3] - q[0] + 1, q[4] - q[1] + 1
                want[m] = c[p0 + (I[m] - q[0]) + nx * ((J[m] - q[1]) + ny * (K[m] - q[2]))]
            assert np.array_equal(pwc[fpos:fpos + n], want)
        fpos += n
    h.close()


@pytest.mark.gpu
def test_improperly_nested_level_is_an_error(cmg):
    # fine box away from the only coarse box
    fi = cmg.FineInterp((0, 0, 0, 31, 31, 31), [(16, 16, 16, 23, 23, 23)], [(0, 0, 0, 7, 7, 7)])
    with pytest.raises(cmg.CmgError) as e:
        fi.interp_to_fine(np.zeros(512))
    assert e.value.code == cmg.CMG_EINVAL and "nested" in str(e.value)
    # piecewise constant needs only the coarsened fine box, not covered either
    with pytest.raises(cmg.CmgError):
        fi.interp_to_fine(np.zeros(512), pwc=True)
    fi.close()
    fi = cmg.FineInterp((0, 0, 0, 31, 31, 31), [(0, 0, 0, 7, 7, 7)], [(0, 0, 0, 3, 3, 3)])
    with pytest.raises(cmg.CmgError):
        fi.interp_to_fine(np.zeros(64))  # grow(b, 1) & domain reaches past the coarse box
    out = fi.interp_to_fine(np.arange(64.0), pwc=True)
    assert out.size == 512 and out[0] == 0.0 and out[-1] == 63.0
    fi.close()


@pytest.mark.gpu
def test_large_boxes_take_the_two_kernel_path(cmg):
    """A fine box whose staging block exceeds shared memory (48^3 fine, 26^3
    coarse staging cells) sends the whole level through the gather kernel and
    the interpolation kernel; both entry points still equal the numpy
    restatement of the reference bit for bit."""
    from test_fineinterp import fine_interp_numpy
    import make_golden_fineinterp as mg
    # in the hierarchy's (sorted) box order, which its data follow
    coarse_boxes = sorted((x, y, z, x + 15, y + 15, z + 15) for z in (0, 16) for y in (0, 16) for x in (0, 16))
    fine_boxes = [(8, 8, 8, 55, 55, 55), (56, 0, 0, 63, 7, 7)]
    c = mg.seeded_field(coarse_boxes, 32, 77)
    want = fine_interp_numpy(coarse_boxes, c, fine_boxes, 32, 0)
    h = cmg.Hierarchy(32, [coarse_boxes, fine_boxes])
    assert h.boxes(0) == coarse_boxes and h.boxes(1) == fine_boxes
    h.set_phi(0, c)
    h.interp_to_fine(1)
    assert np.array_equal(h.phi(1), want)
    h.close()
    fi = cmg.FineInterp((0, 0, 0, 63, 63, 63), fine_boxes, coarse_boxes)
    assert not fi.is_fused()
    assert np.array_equal(fi.interp_to_fine(c), want)
    fi.close()


@pytest.mark.gpu
def test_staging_above_48kb_takes_the_shared_memory_opt_in(cmg):
    """A 40^3 fine box (22^3 coarse staging cells, 85 KB) stays on the one-kernel path with the shared-memory
    opt-in; the output equals the numpy restatement bit for bit."""
    from test_fineinterp import fine_interp_numpy
    import make_golden_fineinterp as mg
    coarse_boxes = sorted((x, y, z, x + 15, y + 15, z + 15) for z in (0, 16) for y in (0, 16) for x in (0, 16))
    fine_boxes = [(8, 8, 8, 47, 47, 47)]
    c = mg.seeded_field(coarse_boxes, 32, 78)
    want = fine_interp_numpy(coarse_boxes, c, fine_boxes, 32, 0)
    h = cmg.Hierarchy(32, [coarse_boxes, fine_boxes])
    h.set_phi(0, c)
    h.interp_to_fine(1)
    assert np.array_equal(h.phi(1), want)
    h.close()
    fi = cmg.FineInterp((0, 0, 0, 63, 63, 63), fine_boxes, coarse_boxes)
    assert fi.is_fused()
    assert np.array_equal(fi.interp_to_fine(c), want)
    assert np.array_equal(fi.interp_to_fine(c, pwc=True), fine_interp_numpy(coarse_boxes, c, fine_boxes, 32, 1))
    fi.close()


@pytest.mark.gpu
def test_device_pointers_in_stream_order(cmg):
    """cmg_fine_interp_run with device pointers (torch tensors): the coarse data are produced on a caller's
    stream and the object runs on that stream (cmg_fine_interp_set_stream), so no synchronisation is needed in
    between; then on the object's own stream after the caller's stream is waited on.  Both equal the host-array
    path bit for bit, on the fused and on the two-kernel path."""
    import torch
    import make_golden_fineinterp as mg
    coarse_boxes = sorted((x, y, z, x + 15, y + 15, z + 15) for z in (0, 16) for y in (0, 16) for x in (0, 16))
    for fine_boxes in ([(8, 8, 8, 39, 39, 39)], [(8, 8, 8, 55, 55, 55), (56, 0, 0, 63, 7, 7)]):
        c = mg.seeded_field(coarse_boxes, 32, 79)
        fi = cmg.FineInterp((0, 0, 0, 63, 63, 63), fine_boxes, coarse_boxes)
        want = fi.interp_to_fine(c)
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            dc = torch.from_numpy(c).to("cuda", non_blocking=False) * 1.0   # produced on s
            df = torch.zeros(fi.nfine, dtype=torch.float64, device="cuda")
        fi.set_stream(s.cuda_stream)
        fi.interp_to_fine_device(dc.data_ptr(), df.data_ptr())
        s.synchronize()
        assert np.array_equal(df.cpu().numpy(), want)
        # back on the object's own stream: the caller finishes its producer first
        fi.set_stream(None)
        with torch.cuda.stream(s):
            dc2 = dc * 1.0
            df2 = torch.zeros_like(df)
        s.synchronize()
        fi.interp_to_fine_device(dc2.data_ptr(), df2.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(df2.cpu().numpy(), want)
        fi.close()
