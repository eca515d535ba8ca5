"""The oracle's P chain with the 8x8 luma transform and its per-macroblock
4x4/8x8 choice, on the CPU.

The reference's encoder codes 4x4 transforms only, so the 8x8 P chain
(orc_p_frame_t8) is pinned piece by piece: with whole-sample vectors the
prediction is the reference picture itself, so every 8x8 block's levels must
be the oracle's forward transform/quantisation of (source - reference), its
reconstruction the reference decoder's own h264d_idct8_add of those levels
onto the reference block, and each 4x4 block's nz word the mask of the 8x8
zig-zag positions CAVLC codes as that block (a zig-zag written here from
the anti-diagonal rule). The choice (orc_t8_choose) is checked against a
numpy restatement with Walsh-Hadamard matrices, and a chosen frame (t8 = 2)
must equal, macroblock by macroblock, the all-4x4 or all-8x8 frame its flag
names.
"""
import numpy as np
import pytest

H4 = np.array([[1, 1, 1, 1], [1, -1, 1, -1], [1, 1, -1, -1], [1, -1, -1, 1]])
H8 = np.kron(np.array([[1, 1], [1, -1]]), H4)


def _zigzag8():
    pos = sorted(((x + y, x if (x + y) % 2 == 0 else y, 8 * y + x) for y in range(8) for x in range(8)))
    # even anti-diagonals run with x rising (up-right), odd ones with y rising (down-left)
    return [p for _, _, p in pos]


def _choose(res):
    r = np.asarray(res, np.int64).reshape(16, 16)
    c4 = sum(int(np.abs(H4 @ r[y:y + 4, x:x + 4] @ H4.T).sum()) >> 1 for y in range(0, 16, 4) for x in range(0, 16, 4))
    c8 = sum((int(np.abs(H8 @ r[y:y + 8, x:x + 8] @ H8.T).sum()) + 2) >> 2 for y in (0, 8) for x in (0, 8))
    return int(c8 < c4)


def test_zigzag_rule_matches_the_table_start():
    # Table 8-13, 8x8 frame scan: the first positions as (x, y)
    zz = _zigzag8()
    assert [(p % 8, p // 8) for p in zz[:10]] == [(0, 0), (1, 0), (0, 1), (0, 2), (1, 1), (2, 0), (3, 0), (2, 1),
                                                 (1, 2), (0, 3)]
    assert sorted(zz) == list(range(64)) and zz[-1] == 63


def test_choice_matches_numpy(oracle_mod):
    rs = np.random.Generator(np.random.PCG64(11))
    cases = [np.zeros((16, 16)), np.full((16, 16), 9), np.full((16, 16), -255), np.tile([[5, -5], [-5, 5]], (8, 8))]
    for k in range(300):
        scale = int(rs.integers(1, 256))
        r = rs.integers(-scale, scale + 1, (16, 16))
        if k % 3 == 0:  # smooth residuals, where 8x8 tends to win
            r = np.cumsum(np.cumsum(rs.integers(-1, 2, (16, 16)), 0), 1)
        cases.append(np.clip(r, -255, 255))
    seen = set()
    for r in cases:
        want = _choose(r)
        assert oracle_mod.t8_choose(r) == want
        seen.add(want)
    assert seen == {0, 1}
    assert oracle_mod.t8_choose(np.zeros((16, 16))) == 0  # equal costs: 4x4
    assert oracle_mod.t8_choose(np.full((16, 16), 9)) == 1


def _pictures(W, H, seed):
    from b200enc import synth
    seq = synth.Sequence(W, H, seed=seed, pan=True)
    (y0, uv0), (y1, uv1) = seq.frame(0), seq.frame(1)
    return [np.ascontiguousarray(a) for a in (y0, uv0, y1, uv1)]


@pytest.mark.parametrize("qp", [0, 18, 27, 40, 51])
def test_8x8_chain_with_whole_sample_vectors(oracle_mod, qp):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    W, H = 96, 64
    y0, uv0, y1, uv1 = _pictures(W, H, qp)
    mbw, mbh = W // 16, H // 16
    mbs = mbw * mbh
    mv = np.zeros((mbs, 4), np.int32)
    f = oracle_mod.frame(W, H, qp)
    rec_y, rec_uv = np.zeros((H, W), np.uint8), np.zeros((H // 2, W), np.uint8)
    o, flags = oracle_mod.p_frame_t8(f, y1, uv1, y0, uv0, mv, rec_y, rec_uv, 1)
    assert (flags == 1).all()
    zz = _zigzag8()
    nz = o["nz"].reshape(mbs, 24).view(np.uint32)
    for mb in range(mbs):
        X, Y = 16 * (mb % mbw), 16 * (mb // mbw)
        lev = o["levels"].reshape(mbs, 384)[mb]
        for q in range(4):
            qx, qy = 8 * (q & 1), 8 * (q >> 1)
            src = y1[Y + qy:Y + qy + 8, X + qx:X + qx + 8].astype(np.int16)
            ref = y0[Y + qy:Y + qy + 8, X + qx:X + qx + 8]
            l8 = lev[64 * q:64 * q + 64]
            np.testing.assert_array_equal(l8, oracle_mod.fwd_quant8((src - ref).reshape(1, 64), qp, 0)[0])
            np.testing.assert_array_equal(rec_y[Y + qy:Y + qy + 8, X + qx:X + qx + 8],
                                          oracle_mod.ref_idct8_add(l8.reshape(1, 64), ref.reshape(1, 8, 8), qp)[0])
            for i in range(4):
                m = sum(1 << j for j in range(16) if l8[zz[4 * j + i]] != 0)
                rb = (qy // 4 + (i >> 1)) * 4 + qx // 4 + (i & 1)
                assert nz[mb, rb] == m
                assert o["dc"].reshape(mbs, 24)[mb, rb] == 0
    # chroma is the 4x4 chain's
    r0y, r0uv = np.zeros_like(rec_y), np.zeros_like(rec_uv)
    o0 = oracle_mod.p_frame(f, y1, uv1, y0, uv0, mv, r0y, r0uv)
    np.testing.assert_array_equal(o["levels"].reshape(mbs, 24, 16)[:, 16:], o0["levels"].reshape(mbs, 24, 16)[:, 16:])
    np.testing.assert_array_equal(rec_uv, r0uv)


@pytest.mark.parametrize("qp", [12, 27, 44])
def test_chosen_frame_is_the_named_chain_per_macroblock(oracle_mod, qp):
    W, H = 160, 96
    y0, uv0, y1, uv1 = _pictures(W, H, 100 + qp)
    mbw, mbh = W // 16, H // 16
    mbs = mbw * mbh
    rs = np.random.Generator(np.random.PCG64(qp))
    mv = np.zeros((mbs, 4), np.int32)
    mv[:, :2] = rs.integers(-40, 41, (mbs, 2))
    f = oracle_mod.frame(W, H, qp)
    outs, recs = {}, {}
    for t8 in (0, 1, 2):
        ry, ruv = np.zeros((H, W), np.uint8), np.zeros((H // 2, W), np.uint8)
        outs[t8] = oracle_mod.p_frame_t8(f, y1, uv1, y0, uv0, mv, ry, ruv, t8)
        recs[t8] = (ry, ruv)
    flags = outs[2][1]
    assert set(np.unique(flags)) == {0, 1}
    np.testing.assert_array_equal(outs[0][1], 0)
    for mb in range(mbs):
        src = outs[int(flags[mb])][0]
        for k in ("levels", "dc", "nz"):
            np.testing.assert_array_equal(outs[2][0][k].reshape(mbs, -1)[mb], src[k].reshape(mbs, -1)[mb])
        X, Y = 16 * (mb % mbw), 16 * (mb // mbw)
        np.testing.assert_array_equal(recs[2][0][Y:Y + 16, X:X + 16], recs[int(flags[mb])][0][Y:Y + 16, X:X + 16])
    np.testing.assert_array_equal(recs[2][1], recs[0][1])
