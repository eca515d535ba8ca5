"""Full-search window staging: the TMA copy (windows inside the reference
plane) and the clamped word loads (picture edges, planes TMA cannot
describe) give the same motion vectors, bit for bit, and both equal the CPU
oracle; the bounded wait for the copy never runs out (the library's error
word stays clear)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STAGE_KNOB = 5  # B200ENC_TUNE_ME_STAGE: 1 word loads, 2 TMA


def _frames(W, H, seed):
    from b200enc import synth
    seq = synth.Sequence(W, H, seed=seed, pan=True, noise_patch=True)
    return seq.frame(0), seq.frame(1)


def _search(gpu, cur, ref, W, H, RW, RH, rng, lam, zt, stage, mb_list=None, flags=0):
    import torch
    L = gpu.lib()
    assert L.b200enc_tune_set(STAGE_KNOB, stage) == 0
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    mv = torch.full((mbs, 4), -7, dtype=torch.int32, device="cuda")
    try:
        if mb_list is None:
            gpu.me_full_search_ex(cur, ref, W, H, RW, RH, rng, lam, zt, mv, flags=flags)
        else:
            lst = torch.tensor(mb_list, dtype=torch.int32, device="cuda")
            cnt = torch.tensor([len(mb_list)], dtype=torch.int32, device="cuda")
            gpu.me_full_search_ex(cur, ref, W, H, RW, RH, rng, lam, zt, mv, lst, cnt, len(mb_list), flags)
        torch.cuda.synchronize()
    finally:
        L.b200enc_tune_set(STAGE_KNOB, 0)
    return mv.cpu().numpy()


@pytest.mark.parametrize("W,H,coded", [(1920, 1080, True), (1280, 720, False), (640, 480, False), (208, 144, False)])
@pytest.mark.parametrize("rng,lam", [(16, 5), (32, 5)])
def test_tma_equals_loads_and_oracle(gpu, oracle_mod, W, H, coded, rng, lam):
    (y0, uv0), (y1, uv1) = _frames(W, H, seed=W * 3 + H + rng)
    ref = gpu.NV12.from_host(y0, uv0)
    cur = gpu.NV12.from_host(y1, uv1)
    RW, RH = (ref.CW, ref.CH) if coded else (W, H)
    for zt in (512, -1):
        a = _search(gpu, cur, ref, W, H, RW, RH, rng, lam, zt, 2, flags=gpu.ME_LOG_INTEGER)
        b = _search(gpu, cur, ref, W, H, RW, RH, rng, lam, zt, 1, flags=gpu.ME_LOG_INTEGER)
        np.testing.assert_array_equal(a, b, err_msg=f"TMA vs loads {W}x{H} R{rng} zt{zt}")
    f = oracle_mod.frame(W, H, 26, coded_clamp=coded)
    ry = np.ascontiguousarray(ref.y.cpu().numpy()[:RH, :RW])
    want = oracle_mod.me_frame(f, np.ascontiguousarray(y1), ry, rng, lam, -1)
    got = _search(gpu, cur, ref, W, H, RW, RH, rng, lam, -1, 0)
    np.testing.assert_array_equal(got, want, err_msg=f"oracle {W}x{H} R{rng}")
    assert gpu.lib().b200enc_me_wait_errors(1) == 0


def test_list_mode_staging(gpu):
    """The persistent list walk reuses one barrier across macroblocks of both
    kinds (interior by TMA, edge by loads): the phase bookkeeping holds over
    a long mixed list."""
    W, H = 1920, 1080
    (y0, uv0), (y1, uv1) = _frames(W, H, seed=11)
    ref = gpu.NV12.from_host(y0, uv0)
    cur = gpu.NV12.from_host(y1, uv1)
    mbs = 120 * 68
    rs = np.random.default_rng(3)
    lst = sorted(rs.choice(mbs, size=3000, replace=False).tolist())
    full = _search(gpu, cur, ref, W, H, 1920, 1088, 32, 5, -1, 2)
    for stage in (2, 1):
        got = _search(gpu, cur, ref, W, H, 1920, 1088, 32, 5, -1, stage, mb_list=lst)
        np.testing.assert_array_equal(got[lst], full[lst], err_msg=f"list stage {stage}")
        rest = np.setdiff1d(np.arange(mbs), lst)
        assert (got[rest] == -7).all()
    assert gpu.lib().b200enc_me_wait_errors(1) == 0


def test_planes_tma_cannot_describe(gpu, oracle_mod):
    """A reference whose base or pitch is not 16-byte aligned is staged by
    loads throughout, with the same result."""
    import torch
    W, H = 640, 360
    (y0, uv0), (y1, uv1) = _frames(W, H, seed=5)
    cur = gpu.NV12.from_host(y1, uv1)
    aligned = gpu.NV12.from_host(y0, uv0)
    want = _search(gpu, cur, aligned, W, H, W, H, 32, 5, -1, 0)
    # pitch 644 (a multiple of 4, not of 16)
    odd = gpu.NV12.from_host(y0, uv0, pitch=644)
    np.testing.assert_array_equal(_search(gpu, cur, odd, W, H, W, H, 32, 5, -1, 0), want)
    # base 4 bytes past a 16-byte boundary
    buf = torch.zeros((aligned.CH + aligned.CH // 2) * aligned.pitch + 16, dtype=torch.uint8, device="cuda")
    view = buf[4:4 + aligned.buf.numel()].view(aligned.buf.shape)
    view.copy_(aligned.buf)

    class Shifted:
        pitch = aligned.pitch

        @staticmethod
        def yp():
            return gpu._vp(view.data_ptr())

    np.testing.assert_array_equal(_search(gpu, cur, Shifted, W, H, W, H, 32, 5, -1, 0), want)
    assert gpu.lib().b200enc_me_wait_errors(1) == 0
