"""Tile deblocking's premise, checked on the CPU with the oracle.

The tile kernel (csrc/deblock.cu, deblock_tile_kernel) deblocks each tile of
macroblocks together with one macroblock of margin on every side, clipped at
the picture, as a picture of its own (raster order; the margin's outer edges
are not filtered), and keeps the tile. That equals whole-picture raster-order
deblocking (clause 8.7; the reference's h264_deblock.c:263-347) on the tile
because a filter's effect does not travel: each sample a tile needs from
outside depends only on samples within one macroblock of it. Here the oracle
deblocks whole pictures and every tile's crop, on random and adversarial
content (small steps that every filter acts on, bS 1/2 everywhere), intra and
inter, QP 20..51, for several tile shapes; every tile must match, and with no
margin on one side tiles must not.
"""
import numpy as np
import pytest


def _content(rs, mbw, mbh, kind):
    CW, CH = 16 * mbw, 16 * mbh
    mbs = mbw * mbh
    if kind == 0:  # textured, quantised
        y = (np.clip(128 + 30 * rs.standard_normal((CH, CW)), 0, 255) // 5 * 5).astype(np.uint8)
        uv = (np.clip(128 + 20 * rs.standard_normal((CH // 2, CW)), 0, 255) // 4 * 4).astype(np.uint8)
        p_nz = 0.4
    elif kind == 1:  # flat 4x4 blocks with small steps
        blk = rs.integers(-12, 13, (CH // 4, CW // 4))
        y = np.clip(128 + np.kron(blk, np.ones((4, 4))) + rs.integers(-1, 2, (CH, CW)), 0, 255).astype(np.uint8)
        cb = rs.integers(-8, 9, (CH // 8, CW // 4))
        uv = np.clip(128 + np.kron(cb, np.ones((4, 4))), 0, 255).astype(np.uint8)
        p_nz = 0.4
    else:  # ramps of tiny steps: every filter acts; dense coefficients (bS 2) or motion (bS 1)
        y = np.clip(128 + rs.integers(-3, 4, (CH, CW)).cumsum(1) // 4, 0, 255).astype(np.uint8)
        uv = np.clip(128 + rs.integers(-3, 4, (CH // 2, CW)).cumsum(0) // 4, 0, 255).astype(np.uint8)
        p_nz = 0.9 if kind == 2 else 0.2
    nz = (rs.integers(0, 1 << 16, (mbs, 24)) * (rs.random((mbs, 24)) < p_nz)).astype(np.uint32)
    mv = np.zeros((mbs, 4), np.int32)
    mv[:, :2] = rs.integers(-9, 10, (mbs, 2))
    return y, uv, nz, mv


def _crop(oracle_mod, y, uv, nz, mv, mbw, mbh, qp, intra, tile, margin):
    """Deblocks the tile (x0, y0, x1, y1) with `margin` macroblocks (l, t, r, b)
    around it as a picture of its own; returns the tile's planes."""
    x0, y0, x1, y1 = tile
    cx0, cy0 = max(0, x0 - margin[0]), max(0, y0 - margin[1])
    cx1, cy1 = min(mbw, x1 + margin[2]), min(mbh, y1 + margin[3])
    sy = y[16 * cy0:16 * cy1, 16 * cx0:16 * cx1].copy()
    suv = uv[8 * cy0:8 * cy1, 16 * cx0:16 * cx1].copy()
    idx = np.array([yy * mbw + xx for yy in range(cy0, cy1) for xx in range(cx0, cx1)])
    oracle_mod.deblock(cx1 - cx0, cy1 - cy0, qp, intra, np.ascontiguousarray(nz[idx]), np.ascontiguousarray(mv[idx]),
                       sy, suv)
    return (sy[16 * (y0 - cy0):16 * (y1 - cy0), 16 * (x0 - cx0):16 * (x1 - cx0)],
            suv[8 * (y0 - cy0):8 * (y1 - cy0), 16 * (x0 - cx0):16 * (x1 - cx0)])


def _tiles(mbw, mbh, tw, th):
    for y0 in range(0, mbh, th):
        for x0 in range(0, mbw, tw):
            yield x0, y0, min(mbw, x0 + tw), min(mbh, y0 + th)


@pytest.mark.parametrize("intra", [0, 1])
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_tiles_with_one_macroblock_margin_match_the_picture(oracle_mod, intra, kind):
    checked = changed = 0
    for c in range(12):
        rs = np.random.Generator(np.random.PCG64(5000 + 97 * c + 13 * kind + intra))
        mbw, mbh = int(rs.integers(3, 14)), int(rs.integers(3, 11))
        qp = int(rs.integers(20, 52))
        y, uv, nz, mv = _content(rs, mbw, mbh, kind)
        wy, wuv = y.copy(), uv.copy()
        oracle_mod.deblock(mbw, mbh, qp, intra, nz, mv, wy, wuv)
        changed += not np.array_equal(wy, y)
        for tw, th in ((1, 1), (2, 2), (3, 5), (8, 4), (8, 8)):
            for t in _tiles(mbw, mbh, tw, th):
                ty, tuv = _crop(oracle_mod, y, uv, nz, mv, mbw, mbh, qp, intra, t, (1, 1, 1, 1))
                x0, y0, x1, y1 = t
                np.testing.assert_array_equal(ty, wy[16 * y0:16 * y1, 16 * x0:16 * x1], err_msg=f"{t} {tw}x{th}")
                np.testing.assert_array_equal(tuv, wuv[8 * y0:8 * y1, 16 * x0:16 * x1], err_msg=f"{t} {tw}x{th}")
                checked += 1
    assert checked > 500
    assert changed >= 8  # the filters act on most of these pictures


@pytest.mark.parametrize("intra", [0, 1])
@pytest.mark.parametrize("side", range(4))
def test_tiles_without_margin_on_one_side_differ(oracle_mod, intra, side):
    """The margin is needed on every side: without it, some tiles differ."""
    rs = np.random.Generator(np.random.PCG64(77 + side + 4 * intra))
    mbw, mbh = 9, 7
    y, uv, nz, mv = _content(rs, mbw, mbh, 2)
    wy, wuv = y.copy(), uv.copy()
    oracle_mod.deblock(mbw, mbh, 40, intra, nz, mv, wy, wuv)
    margin = [1, 1, 1, 1]
    margin[side] = 0
    wrong = 0
    for t in _tiles(mbw, mbh, 2, 2):
        ty, tuv = _crop(oracle_mod, y, uv, nz, mv, mbw, mbh, 40, intra, t, margin)
        x0, y0, x1, y1 = t
        wrong += not (np.array_equal(ty, wy[16 * y0:16 * y1, 16 * x0:16 * x1])
                      and np.array_equal(tuv, wuv[8 * y0:8 * y1, 16 * x0:16 * x1]))
    assert wrong > 0
