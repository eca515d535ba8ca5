"""The deblocking kernel's schedule, checked on the CPU with the oracle.

The kernel filters each macroblock row as a chain V(0), H(0), V(1), H(1), ...
(V: the macroblock's vertical edges, H: its horizontal edges) and lets a
row's H(x) run once the row above has done V(x+1) (all of its row when x is
the last column); vertical edges wait for nothing from the row above. Any
interleaving of the rows under those rules must give exactly the raster-order
result. Random interleavings are drawn (a row whose next step is allowed is
picked at random, so rows run as far ahead as the rules let them) and
applied through the oracle's step function; an order that lets H(x) run
before the row above has done V(x+1) must not match.
"""
import numpy as np
import pytest


def _steps_random(mbw, mbh, rs):
    """A random order of the 2 * mbw * mbh steps (2 * mb + dir) under the
    kernel's rules."""
    pos = [0] * mbh  # next step of each row: 2 * x + dir
    out = []
    total = 2 * mbw * mbh
    while len(out) < total:
        ready = []
        for y in range(mbh):
            p = pos[y]
            if p == 2 * mbw:
                continue
            x, d = p >> 1, p & 1
            if d == 1 and y > 0:
                # the row above has done V(x+1), or all of its row
                need = 2 * (x + 1) + 1 if x + 1 < mbw else 2 * mbw
                if pos[y - 1] < need:
                    continue
            ready.append(y)
        y = ready[rs.integers(len(ready))]
        p = pos[y]
        out.append(2 * (y * mbw + (p >> 1)) + (p & 1))
        pos[y] += 1
    return out


def _steps_too_eager(mbw, mbh):
    """Column by column: H(x, y) before the row above's V(x+1, y-1)."""
    out = []
    for x in range(mbw):
        for y in range(mbh):
            mb = y * mbw + x
            out += [2 * mb, 2 * mb + 1]
    return out


def _case(rs, mbw, mbh, intra, smooth=False):
    CW, CH = 16 * mbw, 16 * mbh
    if smooth:  # flat 4x4 blocks with small steps: the filters act on most lines
        blk = rs.integers(-12, 13, (CH // 4, CW // 4))
        y = np.clip(128 + np.kron(blk, np.ones((4, 4))) + rs.integers(-1, 2, (CH, CW)), 0, 255).astype(np.uint8)
        cb = rs.integers(-8, 9, (CH // 8, CW // 4))
        uv = np.clip(128 + np.kron(cb, np.ones((4, 4))), 0, 255).astype(np.uint8)
    else:
        y = (np.clip(128 + 30 * rs.standard_normal((CH, CW)), 0, 255) // 5 * 5).astype(np.uint8)
        uv = (np.clip(128 + 20 * rs.standard_normal((CH // 2, CW)), 0, 255) // 4 * 4).astype(np.uint8)
    mbs = mbw * mbh
    nz = (rs.integers(0, 1 << 16, (mbs, 24)) * (rs.random((mbs, 24)) < 0.4)).astype(np.uint32)
    mv = np.zeros((mbs, 4), np.int32)
    mv[:, :2] = rs.integers(-9, 10, (mbs, 2))
    return y, uv, nz, mv


@pytest.mark.parametrize("mbw,mbh", [(6, 5), (9, 4), (1, 6), (7, 1)])
@pytest.mark.parametrize("qp,intra", [(30, 1), (45, 1), (33, 0), (45, 0)])
@pytest.mark.parametrize("smooth", [False, True])
def test_random_kernel_orders_match_raster(oracle_mod, mbw, mbh, qp, intra, smooth):
    rs = np.random.Generator(np.random.PCG64(mbw * 100 + mbh * 7 + qp + intra + smooth))
    y, uv, nz, mv = _case(rs, mbw, mbh, intra, smooth)
    wy, wuv = y.copy(), uv.copy()
    oracle_mod.deblock(mbw, mbh, qp, intra, nz, mv, wy, wuv)
    assert not np.array_equal(wy, y)  # the filters do act on this content
    for _ in range(12):
        order = _steps_random(mbw, mbh, rs)
        assert sorted(order) == list(range(2 * mbw * mbh))
        gy, guv = y.copy(), uv.copy()
        oracle_mod.deblock_steps(mbw, mbh, qp, intra, nz, mv, gy, guv, order)
        np.testing.assert_array_equal(gy, wy)
        np.testing.assert_array_equal(guv, wuv)


@pytest.mark.parametrize("qp,intra", [(40, 1), (45, 0)])
def test_order_that_skips_the_rule_differs(oracle_mod, qp, intra):
    rs = np.random.Generator(np.random.PCG64(7 + qp))
    mbw, mbh = 6, 5
    y, uv, nz, mv = _case(rs, mbw, mbh, intra, smooth=True)
    wy, wuv = y.copy(), uv.copy()
    oracle_mod.deblock(mbw, mbh, qp, intra, nz, mv, wy, wuv)
    gy, guv = y.copy(), uv.copy()
    oracle_mod.deblock_steps(mbw, mbh, qp, intra, nz, mv, gy, guv, _steps_too_eager(mbw, mbh))
    assert not (np.array_equal(gy, wy) and np.array_equal(guv, wuv))


def test_step_outside_picture_is_refused(oracle_mod):
    y = np.zeros((16, 16), np.uint8)
    uv = np.zeros((8, 16), np.uint8)
    with pytest.raises(ValueError):
        oracle_mod.deblock_steps(1, 1, 30, 1, np.zeros((1, 24), np.uint32), np.zeros((1, 4), np.int32), y, uv, [2])
