"""b200enc_deblock_noalloc: deblocking for callers that cannot allocate.

Real-time encode threads (a streaming server's per-frame encode, a VA-API
EndPicture under the driver lock) must not call cudaMalloc, which
synchronises the whole device, and plug-ins with a device-memory budget fixed
at start-up may not allocate later; so they cannot hand b200enc_deblock the
scratch it needs. The no-allocation variant keeps that scratch in a fixed
array inside the library. This file checks, through the C ABI, that it
filters exactly like b200enc_deblock with caller scratch, on two calls in a
row (the second reuses the array the first left behind), at the largest
frame the array covers (512 macroblock rows, every word of it in use), and
that frames beyond that limit and bad arguments are refused.

The file name sorts after every other test file, so pytest collects it last:
the entry point's array is process-wide state that outlives the test, and if
this file fails, a run that stops at the first failure (-x) has still run
every other test. The tests do not depend on the order: each call zeroes the
words it uses, so they also pass alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _picture(rs, mbw, mbh):
    CW, CH = mbw * 16, mbh * 16
    y = (np.clip(128 + 35 * rs.standard_normal((CH, CW)), 0, 255) // 6 * 6).astype(np.uint8)
    uv = (np.clip(128 + 25 * rs.standard_normal((CH // 2, CW)), 0, 255) // 4 * 4).astype(np.uint8)
    mbs = mbw * mbh
    nz = (rs.integers(0, 1 << 16, (mbs, 24)) * (rs.random((mbs, 24)) < 0.3)).astype(np.uint32)
    mv = np.zeros((mbs, 4), np.int32)
    mv[:, :2] = rs.integers(-9, 10, (mbs, 2))
    return y, uv, nz, mv


def test_noalloc_deblock_matches_caller_scratch_twice(gpu):
    import torch
    L = gpu.lib()
    stream = torch.cuda.current_stream()
    rs = np.random.Generator(np.random.PCG64(2024))
    for call, (mbw, mbh, qp, intra) in enumerate(((40, 30, 33, 0), (24, 17, 45, 1))):
        y, uv, nz, mv = _picture(rs, mbw, mbh)
        nz_d = torch.from_numpy(nz.view(np.int32)).cuda()
        mv_d = torch.from_numpy(mv).cuda()
        want = gpu.NV12.from_host(y, uv)
        got = gpu.NV12.from_host(y, uv)
        scr = gpu.scratch(mbh)
        gpu.deblock(mbw, mbh, qp, intra, nz_d, mv_d, want, scr)
        assert gpu.wavefront_status(scr) == 0
        rc = L.b200enc_deblock_noalloc(mbw, mbh, qp, intra, ctypes.c_void_p(nz_d.data_ptr()),
                                       ctypes.c_void_p(mv_d.data_ptr()), ctypes.c_void_p(got.y.data_ptr()),
                                       ctypes.c_void_p(got.uv.data_ptr()), got.pitch,
                                       ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, f"call {call}: rc={rc}"
        status = torch.full((1,), 7, dtype=torch.int32).pin_memory()
        assert L.b200enc_deblock_noalloc_status(ctypes.c_void_p(status.data_ptr()),
                                                ctypes.c_void_p(stream.cuda_stream)) == 0
        torch.cuda.synchronize()
        assert int(status[0]) == 0, f"call {call}: status {int(status[0])}"
        assert torch.equal(got.buf, want.buf), f"call {call}: no-alloc deblocking differs"
        assert not torch.equal(got.buf, gpu.NV12.from_host(y, uv).buf), "the filter should change the picture"


def test_noalloc_deblock_at_its_row_limit(gpu):
    import torch
    L = gpu.lib()
    stream = torch.cuda.current_stream()
    rs = np.random.Generator(np.random.PCG64(512))
    mbw, mbh, qp = 1, 512, 36
    y, uv, nz, mv = _picture(rs, mbw, mbh)
    nz_d = torch.from_numpy(nz.view(np.int32)).cuda()
    mv_d = torch.from_numpy(mv).cuda()
    want = gpu.NV12.from_host(y, uv)
    got = gpu.NV12.from_host(y, uv)
    scr = gpu.scratch(mbh)
    gpu.deblock(mbw, mbh, qp, 0, nz_d, mv_d, want, scr)
    assert gpu.wavefront_status(scr) == 0
    for call in range(2):
        if call:
            got = gpu.NV12.from_host(y, uv)
        rc = L.b200enc_deblock_noalloc(mbw, mbh, qp, 0, ctypes.c_void_p(nz_d.data_ptr()),
                                       ctypes.c_void_p(mv_d.data_ptr()), ctypes.c_void_p(got.y.data_ptr()),
                                       ctypes.c_void_p(got.uv.data_ptr()), got.pitch,
                                       ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, f"call {call}: rc={rc}"
        torch.cuda.synchronize()
        assert torch.equal(got.buf, want.buf), f"call {call}: 16x8192 no-alloc deblocking differs"


def test_noalloc_deblock_refuses_frames_beyond_its_scratch(gpu):
    L = gpu.lib()
    p = ctypes.c_void_p(16)
    assert L.b200enc_deblock_noalloc(8, 513, 30, 0, p, p, p, p, 128, None) == -2


def test_noalloc_deblock_rejects_bad_arguments(gpu):
    L = gpu.lib()
    p = ctypes.c_void_p(256)
    assert L.b200enc_deblock_noalloc(8, 0, 30, 0, p, p, p, p, 128, None) == -1
    assert L.b200enc_deblock_noalloc(8, 4, 52, 0, p, p, p, p, 128, None) == -1
    assert L.b200enc_deblock_noalloc(8, 4, -1, 0, p, p, p, p, 128, None) == -1
    assert L.b200enc_deblock_noalloc(0, 4, 30, 0, p, p, p, p, 128, None) == -1
    assert L.b200enc_deblock_noalloc(8, 4, 30, 0, None, p, p, p, 128, None) == -1
    assert L.b200enc_deblock_noalloc(8, 4, 30, 0, p, p, p, p, 64, None) == -1  # pitch below 8 MBs
    assert L.b200enc_deblock_noalloc_status(None, None) == -1
