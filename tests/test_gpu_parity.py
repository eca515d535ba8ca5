"""GPU parity: every stage of libb200enc.so against the CPU oracle, bit-exact.

All calls go through the C-ABI (include/b200enc.h, include/gpu_compute.h).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _frames(W, H, n=2, seed=1, **kw):
    from b200enc import synth
    seq = synth.Sequence(W, H, seed=seed, **kw)
    return [seq.frame(t) for t in range(n)]


def _pad(y, uv, CW, CH):
    return (np.pad(y, ((0, CH - y.shape[0]), (0, CW - y.shape[1])), mode="edge"),
            np.pad(uv, ((0, CH // 2 - uv.shape[0]), (0, CW - uv.shape[1])), mode="edge"))


def _host_rec(rec, CW, CH):
    return rec.y.cpu().numpy()[:CH, :CW].copy(), rec.uv.cpu().numpy()[:CH // 2, :CW].copy()


def _cmp_out(got, want, what, check_mv=True):
    np.testing.assert_array_equal(got["levels"], want["levels"], err_msg=f"{what}: levels")
    np.testing.assert_array_equal(got["dc"], want["dc"], err_msg=f"{what}: dc")
    np.testing.assert_array_equal(got["nz"], want["nz"], err_msg=f"{what}: nz")
    np.testing.assert_array_equal(got["pred_mode"], want["pred_mode"], err_msg=f"{what}: pred_mode")
    if check_mv:
        np.testing.assert_array_equal(got["mv"], want["mv"], err_msg=f"{what}: mv")


SIZES = [(640, 480), (48, 32), (16, 16), (80, 40), (200, 120)]


@pytest.mark.parametrize("W,H", SIZES)
@pytest.mark.parametrize("rng,lam", [(16, 5), (32, 8)])
def test_me_full_search(gpu, oracle_mod, W, H, rng, lam):
    import torch
    (y0, uv0), (y1, uv1) = _frames(W, H, 2, seed=W + H)
    ref = gpu.NV12.from_host(y0, uv0)
    cur = gpu.NV12.from_host(y1, uv1)
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    for zt in (512, -1):
        mv = torch.zeros((mbs, 4), dtype=torch.int32, device="cuda")
        gpu.me_full_search(cur, ref, W, H, W, H, rng, lam, zt, mv)
        torch.cuda.synchronize()
        f = oracle_mod.frame(W, H, 26, coded_clamp=False)
        want = oracle_mod.me_frame(f, np.ascontiguousarray(y1), np.ascontiguousarray(y0), rng, lam, zt)
        np.testing.assert_array_equal(mv.cpu().numpy(), want, err_msg=f"ME {W}x{H} R{rng} zt{zt}")


def test_me_1080p_coded_clamp(gpu, oracle_mod):
    import torch
    W, H = 1920, 1080
    (y0, uv0), (y1, uv1) = _frames(W, H, 2, seed=5, pan=True, noise_patch=True)
    ref = gpu.NV12.from_host(y0, uv0)
    cur = gpu.NV12.from_host(y1, uv1)
    mv = torch.zeros((120 * 68, 4), dtype=torch.int32, device="cuda")
    gpu.me_full_search(cur, ref, W, H, 1920, 1088, 16, 5, 512, mv)
    torch.cuda.synchronize()
    f = oracle_mod.frame(W, H, 26, coded_clamp=True)
    ry, _ = _pad(y0, uv0, 1920, 1088)
    want = oracle_mod.me_frame(f, np.ascontiguousarray(y1), np.ascontiguousarray(ry), 16, 5, 512)
    np.testing.assert_array_equal(mv.cpu().numpy(), want)


@pytest.mark.parametrize("W,H", SIZES + [(1920, 1080)])
@pytest.mark.parametrize("coded_clamp", [True, False])
@pytest.mark.parametrize("qp", [0, 12, 26, 37, 51])
def test_p_frame(gpu, oracle_mod, W, H, coded_clamp, qp):
    import torch
    (y0, uv0), (y1, uv1) = _frames(W, H, 2, seed=W * 3 + qp)
    CW, CH = gpu.coded(W, H)
    RW, RH = (CW, CH) if coded_clamp else (W, H)
    ref = gpu.NV12.from_host(y0, uv0)
    cur = gpu.NV12.from_host(y1, uv1)
    mbs = (CW // 16) * (CH // 16)
    rs = np.random.Generator(np.random.PCG64(qp + W))
    mvh = np.zeros((mbs, 4), np.int32)
    mvh[:, :2] = rs.integers(-70, 71, (mbs, 2))  # every fractional phase, edges beyond the frame
    mv = torch.from_numpy(mvh).cuda()
    out = gpu.Outputs(W, H)
    rec = gpu.NV12(W, H)
    gpu.p_frame(cur, ref, W, H, RW, RH, qp, mv, out, rec)
    torch.cuda.synchronize()
    f = oracle_mod.frame(W, H, qp, coded_clamp=coded_clamp)
    ry, ruv = _pad(y0, uv0, CW, CH)
    rec_y = np.zeros((CH, CW), np.uint8)
    rec_uv = np.zeros((CH // 2, CW), np.uint8)
    want = oracle_mod.p_frame(f, np.ascontiguousarray(y1), np.ascontiguousarray(uv1), ry, ruv, mvh, rec_y, rec_uv)
    got = out.host()
    _cmp_out(got, want, f"P {W}x{H} qp{qp}", check_mv=False)
    gy, guv = _host_rec(rec, CW, CH)
    np.testing.assert_array_equal(gy[:RH, :RW], rec_y[:RH, :RW], err_msg="recon Y")
    np.testing.assert_array_equal(guv[:RH // 2, :RW], rec_uv[:RH // 2, :RW], err_msg="recon UV")


@pytest.mark.parametrize("W,H", SIZES + [(1920, 1080)])
@pytest.mark.parametrize("num_slices", [1, 4, 7])
@pytest.mark.parametrize("qp", [10, 26, 40])
@pytest.mark.parametrize("coded_clamp,corner_check", [(True, True), (False, False), (True, False)])
def test_i_frame(gpu, oracle_mod, W, H, num_slices, qp, coded_clamp, corner_check):
    import torch
    (y0, uv0), = _frames(W, H, 1, seed=W + 7 * qp)
    CW, CH = gpu.coded(W, H)
    RW, RH = (CW, CH) if coded_clamp else (W, H)
    cur = gpu.NV12.from_host(y0, uv0)
    out = gpu.Outputs(W, H)
    rec = gpu.NV12(W, H)
    scr = gpu.scratch(CH // 16)
    gpu.i_frame(cur, W, H, RW, RH, qp, num_slices, out, rec, scr, flags=int(corner_check))
    assert gpu.wavefront_status(scr) == 0
    f = oracle_mod.frame(W, H, qp, num_slices=num_slices, coded_clamp=coded_clamp, corner_check=corner_check)
    rec_y = np.zeros((CH, CW), np.uint8)
    rec_uv = np.zeros((CH // 2, CW), np.uint8)
    want = oracle_mod.i_frame(f, np.ascontiguousarray(y0), np.ascontiguousarray(uv0), rec_y, rec_uv)
    _cmp_out(out.host(), want, f"I {W}x{H} qp{qp} slices{num_slices}")
    gy, guv = _host_rec(rec, CW, CH)
    np.testing.assert_array_equal(gy[:RH, :RW], rec_y[:RH, :RW])
    np.testing.assert_array_equal(guv[:RH // 2, :RW], rec_uv[:RH // 2, :RW])


@pytest.mark.parametrize("mbw,mbh", [(40, 30), (1, 1), (2, 7), (7, 2), (120, 68)])
@pytest.mark.parametrize("qp", [15, 24, 33, 45, 51])
@pytest.mark.parametrize("intra", [0, 1])
def test_deblock(gpu, oracle_mod, mbw, mbh, qp, intra):
    _deblock_case(gpu, oracle_mod, mbw, mbh, qp, intra)


@pytest.mark.parametrize("mbw,mbh,ctas", [(120, 68, 1), (120, 68, 3), (13, 9, 1), (13, 9, 2)])
@pytest.mark.parametrize("intra", [0, 1])
def test_deblock_fewer_ctas_than_groups(gpu, oracle_mod, mbw, mbh, ctas, intra):
    """CTAs that take several row groups by ticket (the ring and progress
    words reset between groups; 13 x 9 ends on a one-row group) filter
    exactly as one CTA per group."""
    _deblock_case(gpu, oracle_mod, mbw, mbh, 33, intra, ctas)


def _deblock_case(gpu, oracle_mod, mbw, mbh, qp, intra, ctas=0):
    import torch
    rs = np.random.Generator(np.random.PCG64(mbw * 1000 + mbh * 10 + qp + intra))
    CW, CH = mbw * 16, mbh * 16
    y = (np.clip(128 + 35 * rs.standard_normal((CH, CW)), 0, 255) // 6 * 6).astype(np.uint8)
    uv = (np.clip(128 + 25 * rs.standard_normal((CH // 2, CW)), 0, 255) // 4 * 4).astype(np.uint8)
    mbs = mbw * mbh
    nz = (rs.integers(0, 1 << 16, (mbs, 24)) * (rs.random((mbs, 24)) < 0.3)).astype(np.uint32)
    mvh = np.zeros((mbs, 4), np.int32)
    mvh[:, :2] = rs.integers(-9, 10, (mbs, 2))
    rec = gpu.NV12.from_host(y, uv)
    scr = gpu.scratch(mbh)
    gpu.deblock(mbw, mbh, qp, intra, torch.from_numpy(nz.view(np.int32)).cuda(), torch.from_numpy(mvh).cuda(), rec, scr,
                ctas=ctas)
    assert gpu.wavefront_status(scr) == 0
    wy, wuv = y.copy(), uv.copy()
    oracle_mod.deblock(mbw, mbh, qp, intra, nz, mvh, wy, wuv)
    gy, guv = _host_rec(rec, CW, CH)
    np.testing.assert_array_equal(gy, wy)
    np.testing.assert_array_equal(guv, wuv)


def test_wavefront_bounded_wait_reports_error(gpu):
    """A row nobody publishes: every wait gives up, the kernel returns and the
    status word says so; the context stays usable."""
    import ctypes
    import torch
    L = gpu.lib()
    mbw, mbh = 8, 6
    rec = gpu.NV12(mbw * 16, mbh * 16)
    scr = gpu.scratch(mbh)
    nz = torch.zeros((mbw * mbh, 24), dtype=torch.int32, device="cuda")
    mv = torch.zeros((mbw * mbh, 4), dtype=torch.int32, device="cuda")
    scr[0] = 1  # ticket starts past the first row group: it is never filtered or published
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.b200enc_deblock_launch(mbw, mbh, 30, 1, ctypes.c_void_p(nz.data_ptr()), ctypes.c_void_p(mv.data_ptr()),
                                  ctypes.c_void_p(rec.y.data_ptr()), ctypes.c_void_p(rec.uv.data_ptr()), rec.pitch,
                                  ctypes.c_void_p(scr.data_ptr()), 0, ctypes.c_uint32(2000), ctypes.c_void_p(stream))
    assert rc == 0
    assert gpu.wavefront_status(scr) == 1
    # the device is still fine afterwards
    scr.zero_()
    gpu.deblock(mbw, mbh, 30, 1, nz, mv, rec, scr)
    assert gpu.wavefront_status(scr) == 0


def test_intra_bounded_wait_reports_error(gpu):
    """The intra wavefront with row 0 left unowned gives up within its
    budget, reports error 1, and the next launch on the context is fine."""
    import ctypes
    import torch
    L = gpu.lib()
    W, H = 96, 64
    cur = gpu.NV12(W, H)
    out = gpu.Outputs(W, H)
    rec = gpu.NV12(W, H)
    scr = gpu.scratch(H // 16)
    scr[0] = 1
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.b200enc_i_frame_launch(p(cur.y), p(cur.uv), cur.pitch, W, H, W, H, 26, 1, p(out.levels), p(out.dc),
                                  p(out.nz), p(out.pred_mode), p(out.mv), p(rec.y), p(rec.uv), rec.pitch, p(scr), 0,
                                  ctypes.c_uint32(2000), 1, stream)
    assert rc == 0
    assert gpu.wavefront_status(scr) == 1
    scr.zero_()
    gpu.i_frame(cur, W, H, W, H, 26, 1, out, rec, scr)
    assert gpu.wavefront_status(scr) == 0
