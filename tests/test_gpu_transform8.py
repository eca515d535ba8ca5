"""GPU parity of the H.264 High-profile 8x8 transform and of deblocking with
8x8-transform macroblocks.

* b200enc_h264_t8_recon (scaling, inverse 8x8, add) against the reference
  decoder's h264d_idct8_add on random levels at every QP - the decoder side,
  pinned to the reference;
* b200enc_h264_t8_forward (forward transform, quantisation, nonzero masks)
  against the oracle at every QP, intra and inter rounding, and the round
  trip forward -> recon against the oracle's;
* b200enc_deblock_tiles_t8 against the reference decoder's deblocking with
  per-macroblock transform_size_8x8_flag, on pictures up to 1080p.
All calls go through the C-ABI.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _recon_gpu(gpu, lev, pred, qp):
    """lev [n][64], pred [n][8][8] -> GPU reconstruction [n][8][8] (blocks side by side in a plane)."""
    import torch
    n = lev.shape[0]
    cols = 16
    rows = (n + cols - 1) // cols
    W, H = cols * 8, rows * 8
    plane = np.zeros((H, W), np.uint8)
    xy = np.zeros((n, 2), np.int32)
    for i in range(n):
        y, x = 8 * (i // cols), 8 * (i % cols)
        plane[y:y + 8, x:x + 8] = pred[i]
        xy[i] = (x, y)
    dp, dl, dxy = (torch.from_numpy(a).cuda() for a in (plane, np.ascontiguousarray(lev, np.int16), xy))
    assert gpu.lib().b200enc_h264_t8_recon(_vp(dl), _vp(dxy), _vp(dp), W, n, qp, None) == 0
    torch.cuda.synchronize()
    out = dp.cpu().numpy()
    return np.stack([out[xy[i, 1]:xy[i, 1] + 8, xy[i, 0]:xy[i, 0] + 8] for i in range(n)])


@pytest.mark.parametrize("qp", list(range(0, 52, 5)) + [51])
def test_recon_matches_reference_decoder(gpu, oracle_mod, qp):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    rs = np.random.Generator(np.random.PCG64(100 + qp))
    n = 200
    lev = (rs.integers(-60, 61, (n, 64)) * (rs.random((n, 64)) < 0.25)).astype(np.int16)
    lev[:40] = (rs.integers(-2000, 2001, (40, 64)) * (rs.random((40, 64)) < 0.1)).astype(np.int16)
    pred = rs.integers(0, 256, (n, 8, 8)).astype(np.uint8)
    np.testing.assert_array_equal(_recon_gpu(gpu, lev, pred, qp), oracle_mod.ref_idct8_add(lev, pred, qp))


@pytest.mark.parametrize("qp", [0, 7, 13, 22, 27, 32, 37, 44, 51])
@pytest.mark.parametrize("intra", [0, 1])
def test_forward_matches_oracle_and_round_trips(gpu, oracle_mod, qp, intra):
    import torch
    rs = np.random.Generator(np.random.PCG64(7 * qp + intra))
    n = 333
    src = rs.integers(0, 256, (n, 8, 8)).astype(np.int16)
    pred = np.clip(src + rs.integers(-60, 61, src.shape), 0, 255).astype(np.uint8)
    res = (src - pred.astype(np.int16)).reshape(n, 64)
    res[:20] = rs.integers(-255, 256, (20, 64))  # the extremes
    dr = torch.from_numpy(np.ascontiguousarray(res)).cuda()
    dl = torch.zeros((n, 64), dtype=torch.int16, device="cuda")
    dnz = torch.zeros(n, dtype=torch.int64, device="cuda")
    assert gpu.lib().b200enc_h264_t8_forward(_vp(dr), _vp(dl), _vp(dnz), n, qp, intra, None) == 0
    torch.cuda.synchronize()
    lev = dl.cpu().numpy()
    want = oracle_mod.fwd_quant8(res, qp, intra)
    np.testing.assert_array_equal(lev, want)
    masks = dnz.cpu().numpy().view(np.uint64)
    exp = ((want != 0).astype(np.uint64) << np.arange(64, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
    np.testing.assert_array_equal(masks, exp)
    np.testing.assert_array_equal(_recon_gpu(gpu, lev, pred, qp), oracle_mod.dequant_idct8_add(lev, pred, qp))


@pytest.mark.parametrize("mbw,mbh", [(1, 1), (13, 9), (120, 68)])
@pytest.mark.parametrize("p8", [0.5, 1.0])
@pytest.mark.parametrize("qp", [28, 40])
def test_tile_deblocking_with_t8_macroblocks(gpu, oracle_mod, mbw, mbh, p8, qp):
    import torch
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    rs = np.random.Generator(np.random.PCG64(mbw + 3 * mbh + int(10 * p8) + qp))
    CW, CH = mbw * 16, mbh * 16
    y = (np.clip(128 + 35 * rs.standard_normal((CH, CW)), 0, 255) // 6 * 6).astype(np.uint8)
    uv = (np.clip(128 + 25 * rs.standard_normal((CH // 2, CW)), 0, 255) // 4 * 4).astype(np.uint8)
    mbs = mbw * mbh
    nz = (rs.integers(0, 1 << 16, (mbs, 24)) * (rs.random((mbs, 24)) < 0.3)).astype(np.uint32)
    mv = np.zeros((mbs, 4), np.int32)
    mv[:, :2] = rs.integers(-9, 10, (mbs, 2))
    t8 = (rs.random(mbs) < p8).astype(np.uint8)
    src = gpu.NV12.from_host(y, uv)
    dst = gpu.NV12(CW, CH)
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    dnz, dt8, dmv = (torch.from_numpy(a).cuda() for a in (nz.view(np.int32), t8, mv))
    assert gpu.lib().b200enc_deblock_tiles_t8(mbw, mbh, qp, 0, _vp(dnz), _vp(dt8), _vp(dmv), src.yp(), src.uvp(),
                                              dst.yp(), dst.uvp(), src.pitch, _vp(st), None) == 0
    torch.cuda.synchronize()
    assert st.cpu().tolist()[:3] == [0, 0, 0]
    wy, wuv = y.copy(), uv.copy()
    oracle_mod.ref_deblock_t8(mbw, mbh, qp, 0, nz, t8, mv, wy, wuv)
    np.testing.assert_array_equal(dst.y.cpu().numpy()[:CH, :CW], wy)
    np.testing.assert_array_equal(dst.uv.cpu().numpy()[:CH // 2, :CW], wuv)
