"""The intra wavefront kernel's schedule, checked on the CPU with the oracle.

The kernel walks each macroblock row left to right and starts macroblock x of
row y once row y-1 has finished its macroblocks 0..x (I16x16 prediction reads
the left, top and top-left reconstruction, never the top-right). Every
interleaving of the rows under that rule must give exactly the raster-order
frame: random ones are drawn (a row whose next macroblock is allowed is picked
at random) and run through the oracle's per-macroblock step; an order that
runs a row before the row above must not match.
"""
import numpy as np
import pytest


def _order_random(mbw, mbh, rs):
    pos = [0] * mbh
    out = []
    while len(out) < mbw * mbh:
        ready = [y for y in range(mbh) if pos[y] < mbw and (y == 0 or pos[y - 1] >= pos[y] + 1)]
        y = ready[rs.integers(len(ready))]
        out.append(y * mbw + pos[y])
        pos[y] += 1
    return out


def _frame_case(oracle_mod, W, H, qp, slices, corner, seed):
    rs = np.random.Generator(np.random.PCG64(seed))
    mbw, mbh = (W + 15) // 16, (H + 15) // 16
    CW, CH = 16 * mbw, 16 * mbh
    base = rs.integers(60, 200, (CH // 8 + 1, CW // 8 + 1)).astype(np.float64)
    y = np.clip(np.kron(base, np.ones((8, 8)))[:CH, :CW] + rs.normal(0, 6, (CH, CW)), 0, 255).astype(np.uint8)
    uv = np.clip(128 + rs.normal(0, 20, (CH // 2, CW)), 0, 255).astype(np.uint8)
    f = oracle_mod.frame(W, H, qp, num_slices=slices, corner_check=corner)
    return f, y, uv, mbw, mbh, CW, CH, rs


def _run(oracle_mod, f, y, uv, CW, CH, order=None):
    ry = np.zeros((CH, CW), np.uint8)
    ruv = np.zeros((CH // 2, CW), np.uint8)
    if order is None:
        o = oracle_mod.i_frame(f, y, uv, ry, ruv)
    else:
        o = oracle_mod.i_frame_steps(f, y, uv, ry, ruv, order)
    return o, ry, ruv


@pytest.mark.parametrize("W,H", [(96, 80), (160, 48), (16, 96), (200, 120)])
@pytest.mark.parametrize("qp,slices,corner", [(26, 1, True), (40, 3, True), (12, 2, False)])
def test_random_wavefront_orders_match_raster(oracle_mod, W, H, qp, slices, corner):
    f, y, uv, mbw, mbh, CW, CH, rs = _frame_case(oracle_mod, W, H, qp, slices, corner, W * 7 + H + qp + slices)
    want, wy, wuv = _run(oracle_mod, f, y, uv, CW, CH)
    for _ in range(8):
        order = _order_random(mbw, mbh, rs)
        assert sorted(order) == list(range(mbw * mbh))
        got, gy, guv = _run(oracle_mod, f, y, uv, CW, CH, order)
        for k in ("levels", "dc", "nz", "pred_mode"):
            np.testing.assert_array_equal(got[k], want[k], err_msg=k)
        np.testing.assert_array_equal(gy, wy)
        np.testing.assert_array_equal(guv, wuv)


def test_row_before_the_row_above_differs(oracle_mod):
    f, y, uv, mbw, mbh, CW, CH, _ = _frame_case(oracle_mod, 96, 80, 26, 1, True, 5)
    want, wy, _ = _run(oracle_mod, f, y, uv, CW, CH)
    order = [r * mbw + x for r in reversed(range(mbh)) for x in range(mbw)]  # bottom row first
    got, gy, _ = _run(oracle_mod, f, y, uv, CW, CH, order)
    assert not (np.array_equal(gy, wy) and np.array_equal(got["levels"], want["levels"]))


def test_macroblock_outside_picture_is_refused(oracle_mod):
    f, y, uv, mbw, mbh, CW, CH, _ = _frame_case(oracle_mod, 32, 32, 26, 1, True, 1)
    with pytest.raises(ValueError):
        _run(oracle_mod, f, y, uv, CW, CH, [0, 1, 2, 3, 4])
