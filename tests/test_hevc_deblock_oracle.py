"""The reference's HEVC deblocking filter as the tests drive it
(oracle/_ref/libhevcfilt.so: the decoder's hevc_filter.c behind
oracle/hevc_filter_shim.c), on the CPU: it filters a blocky picture at high
QP, leaves it alone where the standard says nothing is filtered (QP below
the tables' first non-zero entries, every slice disabled, no slice
settings), keeps lossless blocks and the stride padding untouched."""
import os

import numpy as np
import pytest

import hevc_db_inputs as hdi

needs_ref = pytest.mark.skipif(not os.path.exists(hdi.FILT_SO), reason="reference HEVC filter not built")


@pytest.fixture(scope="module")
def b2():
    import b200enc
    return b200enc


def _changed(a, b):
    return int(sum(int((x != y).sum()) for x, y in zip(a, b)))


@needs_ref
@pytest.mark.parametrize("bit_depth", [8, 10])
def test_reference_filters_blocky_picture(b2, bit_depth):
    case = hdi.make_case(1, 128, 64, bit_depth=bit_depth, log2_ctb=5, qp_range=(34, 51))
    out = hdi.reference(b2, case)
    assert _changed(out, case["planes"]) > 500
    for c, (o, i) in enumerate(zip(out, case["planes"])):
        w = case["width"] >> (1 if c else 0)
        np.testing.assert_array_equal(o[:, w:], i[:, w:])          # padding untouched


@needs_ref
def test_reference_low_qp_leaves_picture(b2):
    case = hdi.make_case(2, 96, 48, qp_range=(0, 15), slice_params=[(0, 0, 0, 1)])
    assert _changed(hdi.reference(b2, case), case["planes"]) == 0


@needs_ref
def test_reference_disabled_or_missing_slice_settings(b2):
    case = hdi.make_case(3, 96, 64, qp_range=(40, 51), slices=2, log2_ctb=4,
                         slice_params=[(0, 0, 1, 1), (0, 0, 1, 0)])
    assert _changed(hdi.reference(b2, case), case["planes"]) == 0
    assert _changed(hdi.reference(b2, case, slice_filter=None), case["planes"]) == 0


@needs_ref
def test_reference_keeps_lossless_blocks(b2):
    case = hdi.make_case(4, 128, 64, qp_range=(40, 51), lossless=0.3, log2_min_cb=3)
    out = hdi.reference(b2, case)
    nf = case["no_filter"]
    ys, xs = np.nonzero(nf)
    assert len(ys) > 0 and _changed(out, case["planes"]) > 0
    for y, x in zip(ys, xs):
        np.testing.assert_array_equal(out[0][8 * y:8 * y + 8, 8 * x:8 * x + 8],
                                      case["planes"][0][8 * y:8 * y + 8, 8 * x:8 * x + 8])
        for c in (1, 2):
            np.testing.assert_array_equal(out[c][4 * y:4 * y + 4, 4 * x:4 * x + 4],
                                          case["planes"][c][4 * y:4 * y + 4, 4 * x:4 * x + 4])


def test_parameter_block_layout(b2):
    """The ctypes parameter block and record dtypes have the layout of
    include/b200enc.h, which csrc/hevc_deblock.cu pins with static_asserts
    (168 bytes, edges at 64, qp_y at 104, tile_of_ctb at 144)."""
    P = b2.HevcDeblockParams
    assert b2.HEVC_MVF.itemsize == 20 and b2.HEVC_SLICE_FILTER.itemsize == 8
    assert (P.edges.offset, P.qp_y.offset, P.tile_of_ctb.offset) == (64, 104, 144)
    assert __import__("ctypes").sizeof(P) == 168
