"""HEVC deblocking on the GPU (csrc/hevc_deblock.cu, b200enc_hevc_deblock)
against the reference decoder's loop filter (hevc_filter.c compiled in
oracle/_ref/libhevcfilt.so), bit for bit over the whole buffers (the stride
padding included): 8- and 10-bit pictures from 200x136 to 3840x2160, CTB
16/32/64, min CB 8/16, several slices with their own beta/tC offsets,
disabled and not-across-slices ones, tiles with and without filtering
across them, lossless blocks, chroma QP offsets, intra pictures (no motion
field: bS 2 everywhere), and the inputs under which nothing may change."""
import os

import numpy as np
import pytest

import hevc_db_inputs as hdi

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not os.path.exists(hdi.FILT_SO), reason="reference HEVC filter not built")


def _dev(a):
    import torch
    if a is None:
        return None
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()


def _run_gpu(gpu, case, slice_filter="default"):
    import torch
    planes = [_dev(p) for p in case["planes"]]
    bufs = {k: _dev(case[k]) for k in ("edges", "mvf", "cbf", "qp_y", "no_filter", "slice_of_ctb", "tile_of_ctb")}
    sf = case["slice_filter"] if slice_filter == "default" else slice_filter
    dcase = dict(case, **bufs)
    q = hdi.params(gpu, dcase, lambda t: t.data_ptr(), planes=planes, slice_filter=None)
    sfd = _dev(sf)
    if sf is not None:
        q.slice_filter, q.n_slice_filter = sfd.data_ptr(), len(sf)
    gpu.hevc_deblock(q)
    torch.cuda.synchronize()
    out = []
    for t, p in zip(planes, case["planes"]):
        out.append(t.cpu().numpy().view(p.dtype).reshape(p.shape))
    return out


CASES = {
    "1080p_8bit": dict(seed=11, width=1920, height=1080, bit_depth=8, log2_ctb=6, log2_min_cb=3),
    "multi_10bit": dict(seed=12, width=416, height=240, bit_depth=10, log2_ctb=5, log2_min_cb=3, slices=3, tiles=2,
                        lossless=0.1, cb_qp_offset=-5, cr_qp_offset=7, qp_range=(-12, 51)),
    "odd_8bit_ctb16": dict(seed=13, width=200, height=136, bit_depth=8, log2_ctb=4, log2_min_cb=3, slices=2,
                           tiles=3, across_tiles=True, cb_qp_offset=12, cr_qp_offset=-12),
    "intra_8bit": dict(seed=14, width=640, height=480, bit_depth=8, log2_ctb=6, log2_min_cb=4, intra=True),
    "intra_10bit_tiles": dict(seed=15, width=352, height=288, bit_depth=10, log2_ctb=5, log2_min_cb=4, intra=True,
                              tiles=2, slices=2, qp_range=(-12, 51)),
    "uhd_10bit": dict(seed=16, width=3840, height=2160, bit_depth=10, log2_ctb=6, log2_min_cb=3, slices=4),
}


@needs_ref
@pytest.mark.parametrize("name", list(CASES))
def test_hevc_deblock_matches_reference(gpu, name):
    case = hdi.make_case(**CASES[name])
    want = hdi.reference(gpu, case)
    changed = sum(int((w != p).sum()) for w, p in zip(want, case["planes"]))
    assert changed > 0, "the case filters nothing: it would not test the filter"
    got = _run_gpu(gpu, case)
    for c in range(3):
        np.testing.assert_array_equal(got[c], want[c], err_msg=f"{name} plane {c}")


@needs_ref
def test_hevc_deblock_nothing_to_do(gpu):
    """No slice settings, every slice disabled, or QP under the tables'
    first non-zero entries: the picture is returned as it was."""
    case = hdi.make_case(21, 256, 128, qp_range=(40, 51))
    for c, g in zip(case["planes"], _run_gpu(gpu, case, slice_filter=None)):
        np.testing.assert_array_equal(g, c)
    case = hdi.make_case(22, 256, 128, qp_range=(40, 51), slices=2, log2_ctb=5,
                         slice_params=[(0, 0, 1, 1), (4, 4, 1, 0)])
    for c, g in zip(case["planes"], _run_gpu(gpu, case)):
        np.testing.assert_array_equal(g, c)
    case = hdi.make_case(23, 256, 128, qp_range=(0, 15), slice_params=[(0, 0, 0, 1)])
    for c, g in zip(case["planes"], _run_gpu(gpu, case)):
        np.testing.assert_array_equal(g, c)


def test_hevc_deblock_rejects_bad_parameters(gpu):
    """Parameters the filter cannot take are refused before any launch."""
    import ctypes
    case = hdi.make_case(31, 64, 32)
    L = gpu.lib()
    planes = [_dev(p) for p in case["planes"]]
    bufs = {k: _dev(case[k]) for k in ("edges", "mvf", "cbf", "qp_y")}
    sfd = _dev(case["slice_filter"])
    base = hdi.params(gpu, dict(case, **bufs), lambda t: t.data_ptr(), planes=planes, slice_filter=None)
    base.slice_filter, base.n_slice_filter = sfd.data_ptr(), 1
    for field, value in (("bit_depth_luma", 12), ("width", 60), ("log2_ctb", 7), ("edges_stride", 4),
                         ("min_pu_width", 8), ("qp_y", None), ("log2_min_cb", 2)):
        q = gpu.HevcDeblockParams.from_buffer_copy(base)
        setattr(q, field, value)
        assert L.b200enc_hevc_deblock(ctypes.byref(q), None) == -1, field
    assert L.b200enc_hevc_deblock(None, None) == -1
