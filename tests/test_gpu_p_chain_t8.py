"""GPU parity of the P chain with the 8x8 luma transform (b200enc_p_frame_t8)
against the oracle (orc_p_frame_t8): every macroblock 8x8 (t8 = 1) or the
4x4/8x8 choice per macroblock (t8 = 2) - levels, DC words, nz masks, the
per-macroblock flags and the reconstruction, bit-exact, with vectors of
every fractional phase reaching past the picture, through the C-ABI.
"""
import numpy as np
import pytest

from test_gpu_parity import _frames, _host_rec, _pad

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("W,H", [(48, 32), (200, 120), (640, 480), (1920, 1080)])
@pytest.mark.parametrize("qp", [0, 17, 27, 38, 51])
@pytest.mark.parametrize("t8", [1, 2])
def test_p_frame_t8(gpu, oracle_mod, W, H, qp, t8):
    import torch
    (y0, uv0), (y1, uv1) = _frames(W, H, 2, seed=W + 7 * qp + t8, pan=True)
    CW, CH = gpu.coded(W, H)
    ref = gpu.NV12.from_host(y0, uv0)
    cur = gpu.NV12.from_host(y1, uv1)
    mbs = (CW // 16) * (CH // 16)
    rs = np.random.Generator(np.random.PCG64(qp + W + t8))
    mvh = np.zeros((mbs, 4), np.int32)
    mvh[:, :2] = rs.integers(-70, 71, (mbs, 2))
    mvh[: mbs // 4, :2] = 0  # whole-sample blocks too
    mv = torch.from_numpy(mvh).cuda()
    out = gpu.Outputs(W, H)
    rec = gpu.NV12(W, H)
    flags = torch.full((mbs,), 7, dtype=torch.uint8, device="cuda")
    gpu.p_frame_t8(cur, ref, W, H, CW, CH, qp, mv, out, rec, t8, flags)
    torch.cuda.synchronize()
    f = oracle_mod.frame(W, H, qp)
    ry, ruv = _pad(y0, uv0, CW, CH)
    rec_y = np.zeros((CH, CW), np.uint8)
    rec_uv = np.zeros((CH // 2, CW), np.uint8)
    want, wflags = oracle_mod.p_frame_t8(f, np.ascontiguousarray(y1), np.ascontiguousarray(uv1), ry, ruv, mvh, rec_y,
                                         rec_uv, t8)
    got = out.host()
    for k in ("levels", "dc", "nz", "pred_mode"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=f"t8={t8} {W}x{H} qp{qp}: {k}")
    np.testing.assert_array_equal(flags.cpu().numpy(), wflags, err_msg="per-macroblock choice")
    gy, guv = _host_rec(rec, CW, CH)
    np.testing.assert_array_equal(gy, rec_y, err_msg="recon Y")
    np.testing.assert_array_equal(guv, rec_uv, err_msg="recon UV")
    if t8 == 2 and W >= 200:
        assert 0 < int(wflags.sum()) < mbs  # both sizes chosen somewhere


def test_p_frame_t8_rejects_bad_mode(gpu):
    import torch
    W = H = 32
    f = gpu.NV12(W, H)
    out = gpu.Outputs(W, H)
    mv = torch.zeros((4, 4), dtype=torch.int32, device="cuda")
    L = gpu.lib()
    for bad in (-1, 3):
        assert L.b200enc_p_frame_t8(f.yp(), f.uvp(), f.pitch, f.yp(), f.uvp(), f.pitch, W, H, W, H, 26,
                                    gpu._p(mv), gpu._p(out.levels), gpu._p(out.dc), gpu._p(out.nz),
                                    gpu._p(out.pred_mode), f.yp(), f.uvp(), f.pitch, bad, None, None) == -1
