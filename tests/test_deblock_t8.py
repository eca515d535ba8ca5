"""Deblocking with 8x8-transform macroblocks, on the CPU.

H.264 High profile lets a macroblock code its luma with the 8x8 transform
(transform_size_8x8_flag): its odd internal luma edges are then not filtered
and a boundary strength's coefficient test looks at the 8x8 block
(A1/src/h264_deblock.c:119-137, 294, 324). The oracle's restatement
(orc_deblock_frame_t8) is pinned to the reference decoder's own deblocking
(oracle/_ref/libh264ref.so) on random and adversarial P pictures with random
per-macroblock flags, and the tile premise of the GPU kernel (a tile with
one macroblock of margin deblocked on its own reproduces the picture) is
checked to hold with such macroblocks too.
"""
import numpy as np
import pytest

from test_deblock_tiles import _content, _crop, _tiles


def _t8(rs, mbs, p):
    return (rs.random(mbs) < p).astype(np.uint8)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
@pytest.mark.parametrize("p8", [0.0, 0.5, 1.0])
def test_oracle_t8_matches_reference_decoder(oracle_mod, kind, p8):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    for c in range(6):
        rs = np.random.Generator(np.random.PCG64(700 + 31 * c + 7 * kind + int(10 * p8)))
        mbw, mbh = int(rs.integers(2, 12)), int(rs.integers(2, 9))
        qp = int(rs.integers(20, 52))
        y, uv, nz, mv = _content(rs, mbw, mbh, kind)
        t8 = _t8(rs, mbw * mbh, p8)
        gy, guv = y.copy(), uv.copy()
        oracle_mod.deblock_t8(mbw, mbh, qp, 0, nz, t8, mv, gy, guv)
        wy, wuv = y.copy(), uv.copy()
        oracle_mod.ref_deblock_t8(mbw, mbh, qp, 0, nz, t8, mv, wy, wuv)
        np.testing.assert_array_equal(gy, wy)
        np.testing.assert_array_equal(guv, wuv)
        if p8 == 0.0:  # no 8x8 macroblock: the plain deblocking
            py, puv = y.copy(), uv.copy()
            oracle_mod.deblock(mbw, mbh, qp, 0, nz, mv, py, puv)
            np.testing.assert_array_equal(gy, py)


def test_t8_changes_the_result(oracle_mod):
    rs = np.random.Generator(np.random.PCG64(4))
    mbw, mbh = 8, 6
    y, uv, nz, mv = _content(rs, mbw, mbh, 2)
    a, b = (y.copy(), uv.copy()), (y.copy(), uv.copy())
    oracle_mod.deblock_t8(mbw, mbh, 40, 0, nz, np.zeros(mbw * mbh, np.uint8), mv, *a)
    oracle_mod.deblock_t8(mbw, mbh, 40, 0, nz, np.ones(mbw * mbh, np.uint8), mv, *b)
    assert not np.array_equal(a[0], b[0])


def _crop_t8(oracle_mod, y, uv, nz, t8, mv, mbw, mbh, qp, tile):
    x0, y0, x1, y1 = tile
    cx0, cy0, cx1, cy1 = max(0, x0 - 1), max(0, y0 - 1), min(mbw, x1 + 1), min(mbh, y1 + 1)
    sy = y[16 * cy0:16 * cy1, 16 * cx0:16 * cx1].copy()
    suv = uv[8 * cy0:8 * cy1, 16 * cx0:16 * cx1].copy()
    idx = np.array([yy * mbw + xx for yy in range(cy0, cy1) for xx in range(cx0, cx1)])
    oracle_mod.deblock_t8(cx1 - cx0, cy1 - cy0, qp, 0, np.ascontiguousarray(nz[idx]), np.ascontiguousarray(t8[idx]),
                          np.ascontiguousarray(mv[idx]), sy, suv)
    return (sy[16 * (y0 - cy0):16 * (y1 - cy0), 16 * (x0 - cx0):16 * (x1 - cx0)],
            suv[8 * (y0 - cy0):8 * (y1 - cy0), 16 * (x0 - cx0):16 * (x1 - cx0)])


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_tiles_with_t8_macroblocks_match_the_picture(oracle_mod, kind):
    for c in range(8):
        rs = np.random.Generator(np.random.PCG64(900 + 13 * c + kind))
        mbw, mbh = int(rs.integers(3, 13)), int(rs.integers(3, 10))
        qp = int(rs.integers(20, 52))
        y, uv, nz, mv = _content(rs, mbw, mbh, kind)
        t8 = _t8(rs, mbw * mbh, 0.5)
        wy, wuv = y.copy(), uv.copy()
        oracle_mod.deblock_t8(mbw, mbh, qp, 0, nz, t8, mv, wy, wuv)
        for tw, th in ((1, 1), (3, 2), (8, 8)):
            for t in _tiles(mbw, mbh, tw, th):
                ty, tuv = _crop_t8(oracle_mod, y, uv, nz, t8, mv, mbw, mbh, qp, t)
                x0, y0, x1, y1 = t
                np.testing.assert_array_equal(ty, wy[16 * y0:16 * y1, 16 * x0:16 * x1])
                np.testing.assert_array_equal(tuv, wuv[8 * y0:8 * y1, 16 * x0:16 * x1])
