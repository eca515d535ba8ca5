"""GPU parity of the tile deblocking (b200enc_deblock_tiles) against the oracle.

Every tile shape the autotuner may pick (1..8 x 1..8 macroblocks) must give
the oracle's whole-picture raster-order result bit for bit, intra and inter,
on pictures from one macroblock to 2160p. All calls go through the C-ABI.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TILE_W, TILE_H = 6, 7  # B200ENC_TUNE_DEBLOCK_TILE_W / _H


def _case(rs, mbw, mbh):
    CW, CH = mbw * 16, mbh * 16
    y = (np.clip(128 + 35 * rs.standard_normal((CH, CW)), 0, 255) // 6 * 6).astype(np.uint8)
    uv = (np.clip(128 + 25 * rs.standard_normal((CH // 2, CW)), 0, 255) // 4 * 4).astype(np.uint8)
    mbs = mbw * mbh
    nz = (rs.integers(0, 1 << 16, (mbs, 24)) * (rs.random((mbs, 24)) < 0.3)).astype(np.uint32)
    mv = np.zeros((mbs, 4), np.int32)
    mv[:, :2] = rs.integers(-9, 10, (mbs, 2))
    return y, uv, nz, mv


def _run(gpu, oracle_mod, mbw, mbh, qp, intra, seed=0):
    import torch
    rs = np.random.Generator(np.random.PCG64(seed + mbw * 1000 + mbh * 10 + qp + intra))
    y, uv, nz, mv = _case(rs, mbw, mbh)
    src = gpu.NV12.from_host(y, uv)
    dst = gpu.NV12(mbw * 16, mbh * 16)
    dst.buf.fill_(7)
    status = torch.full((4,), -1, dtype=torch.int32, device="cuda")
    gpu.deblock_tiles(mbw, mbh, qp, intra, torch.from_numpy(nz.view(np.int32)).cuda(), torch.from_numpy(mv).cuda(),
                      src, dst, status)
    torch.cuda.synchronize()
    assert status.cpu().tolist()[:3] == [0, 0, 0]
    wy, wuv = y.copy(), uv.copy()
    oracle_mod.deblock(mbw, mbh, qp, intra, nz, mv, wy, wuv)
    CW, CH = mbw * 16, mbh * 16
    np.testing.assert_array_equal(dst.y.cpu().numpy()[:CH, :CW], wy)
    np.testing.assert_array_equal(dst.uv.cpu().numpy()[:CH // 2, :CW], wuv)
    # the source planes are left as they were
    np.testing.assert_array_equal(src.y.cpu().numpy()[:CH, :CW], y)


@pytest.fixture
def tile_shape(gpu):
    L = gpu.lib()

    def set_shape(tw, th):
        assert L.b200enc_tune_set(TILE_W, tw) == 0 and L.b200enc_tune_set(TILE_H, th) == 0

    yield set_shape
    set_shape(0, 0)


@pytest.mark.parametrize("mbw,mbh", [(1, 1), (3, 2), (13, 9), (120, 68), (240, 135)])
@pytest.mark.parametrize("qp", [22, 33, 45, 51])
@pytest.mark.parametrize("intra", [0, 1])
def test_deblock_tiles_default_shape(gpu, oracle_mod, mbw, mbh, qp, intra):
    _run(gpu, oracle_mod, mbw, mbh, qp, intra)


@pytest.mark.parametrize("tw,th", [(1, 1), (2, 3), (3, 5), (8, 4), (4, 8), (5, 8), (8, 1), (7, 7), (12, 8), (16, 8),
                                   (16, 1), (11, 6)])
@pytest.mark.parametrize("mbw,mbh", [(13, 9), (120, 68)])
@pytest.mark.parametrize("intra", [0, 1])
def test_deblock_tiles_every_shape(gpu, oracle_mod, tile_shape, tw, th, mbw, mbh, intra):
    tile_shape(tw, th)
    _run(gpu, oracle_mod, mbw, mbh, 40, intra, seed=tw * 10 + th)


def test_deblock_tiles_rejects_overlap_and_bad_arguments(gpu):
    import torch
    L = gpu.lib()
    mbw, mbh = 4, 3
    a = gpu.NV12(mbw * 16, mbh * 16)
    b = gpu.NV12(mbw * 16, mbh * 16)
    nz = torch.zeros((mbw * mbh, 24), dtype=torch.int32, device="cuda")
    mv = torch.zeros((mbw * mbh, 4), dtype=torch.int32, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def call(src, dst, pitch=a.pitch, qp=30, status=st, h=mbh):
        return L.b200enc_deblock_tiles(mbw, h, qp, 0, vp(nz), vp(mv), vp(src.y), vp(src.uv), vp(dst.y), vp(dst.uv),
                                       pitch, vp(status) if status is not None else None, None)

    assert call(a, b) == 0
    assert call(a, a) == -1          # in place
    assert call(a, b, qp=52) == -1
    assert call(a, b, pitch=a.pitch - 8) == -1
    assert call(a, b, status=None) == -1
    assert call(a, b, h=0) == -1
    torch.cuda.synchronize()
