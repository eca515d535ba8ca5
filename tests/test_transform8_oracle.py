"""The oracle's 8x8 transform (H.264 High profile), on the CPU.

The decoder side - flat-list scaling, the clause 8.5.13.2 inverse transform
and the add onto the prediction - is pinned to the reference decoder's
h264d_idct8_add (A1/src/h264_recon.c:191) on random levels, including large
ones, at every QP. The encoder side (forward transform and quantisation) has
no reference counterpart: the reference's encoder codes 4x4 transforms only.
Its check is the round trip: at QP 0 the reconstruction is within one step
of the source, and the error grows with QP as the quantiser step does.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("qp", list(range(0, 52, 3)) + [51])
def test_dequant_idct8_matches_reference_decoder(oracle_mod, qp):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    rs = np.random.Generator(np.random.PCG64(qp))
    n = 64
    lev = (rs.integers(-40, 41, (n, 64)) * (rs.random((n, 64)) < 0.3)).astype(np.int16)
    lev[: n // 4] = (rs.integers(-2000, 2001, (n // 4, 64)) * (rs.random((n // 4, 64)) < 0.1)).astype(np.int16)
    pred = rs.integers(0, 256, (n, 8, 8)).astype(np.uint8)
    np.testing.assert_array_equal(oracle_mod.dequant_idct8_add(lev, pred, qp), oracle_mod.ref_idct8_add(lev, pred, qp))


@pytest.mark.parametrize("intra", [0, 1])
def test_forward_quant_round_trip(oracle_mod, intra):
    rs = np.random.Generator(np.random.PCG64(11 + intra))
    src = rs.integers(0, 256, (32, 8, 8)).astype(np.int16)
    pred = np.clip(src + rs.integers(-40, 41, src.shape), 0, 255).astype(np.uint8)
    res = src - pred.astype(np.int16)
    errs = []
    for qp in (0, 12, 24, 36, 51):
        lev = oracle_mod.fwd_quant8(res, qp, intra)
        rec = oracle_mod.dequant_idct8_add(lev, pred, qp)
        errs.append(np.abs(rec.astype(int) - src).mean())
        if qp == 0:
            assert np.abs(rec.astype(int) - src).max() <= 1
    assert errs == sorted(errs)  # coarser quantisation, larger error
