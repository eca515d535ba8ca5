"""Encode -> decode round trip of the reference pipeline on the CPU.

The reference's unchanged host encoder runs over oracle/cpu_boundary.c (the
gpu_compute_* boundary implemented with the CPU oracle, built into
oracle/_ref/libh264enc_cpu.so); its stream is decoded by the reference's
h264dec and every decoded frame must equal the reconstruction the boundary
kept. The GPU twin of this test is tests/test_gpu_roundtrip.py; this one runs
without a GPU, so the stage math and the host encoder's use of it are
checked on every CPU run."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENC_SO = os.path.join(ROOT, "oracle", "_ref", "libh264enc_cpu.so")
DEC = os.path.join(ROOT, "oracle", "_ref", "h264dec")


def encode_cpu(W, H, frames, qp, profile, slices, gop, path, seed=3):
    import b200enc
    from b200enc import synth
    os.environ.update(BC250_FORCE_QP=str(qp), BC250_FORCE_TIER="0", BC250_SLICES_PER_FRAME=str(slices),
                      BC250_FORCE_SLICES="0")
    enc = ctypes.CDLL(ENC_SO)
    ctx = b200enc.GpuContext()
    assert enc.bc250_gpu_init(ctypes.byref(ctx)) == 0
    enc.h264_encoder_create.restype = ctypes.c_void_p
    enc.h264_encoder_create.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_int]
    e = enc.h264_encoder_create(ctypes.byref(ctx), W, H, 30, 8_000_000, profile)
    enc.h264_encoder_set_gop_size(ctypes.c_void_p(e), ctypes.c_uint32(gop))
    enc.h264_encoder_encode_frame_ext.argtypes = [ctypes.c_void_p, ctypes.c_void_p, b200enc.GpuImage,
                                                  b200enc.GpuMemory, ctypes.c_void_p, ctypes.c_size_t]
    img, mem = b200enc.GpuImage(), b200enc.GpuMemory()
    assert enc.gpu_compute_create_image(ctypes.byref(ctx), W, H, 0, ctypes.byref(img), ctypes.byref(mem)) == 0
    seq = synth.Sequence(W, H, seed=seed, pan=True)
    out = np.zeros(W * H * 4, np.uint8)
    stream, recons = bytearray(), []
    CH = (H + 15) // 16 * 16
    for t in range(frames):
        y, uv = seq.frame(t)
        enc.gpu_compute_upload_nv12(ctypes.byref(ctx), ctypes.byref(img), mem, ctypes.c_void_p(y.ctypes.data), W,
                                    ctypes.c_void_p(uv.ctypes.data), W, W, H)
        n = enc.h264_encoder_encode_frame_ext(ctypes.c_void_p(e), ctypes.byref(ctx), img, mem,
                                              ctypes.c_void_p(out.ctypes.data), out.nbytes)
        assert n > 0
        stream += out[:n].tobytes()
        yp, uvp, pitch = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int()
        assert enc.cpu_boundary_recon(ctypes.byref(ctx), ctypes.byref(yp), ctypes.byref(uvp), ctypes.byref(pitch)) == 0
        ry = np.ctypeslib.as_array((ctypes.c_uint8 * (CH * pitch.value)).from_address(yp.value)).reshape(CH, pitch.value)
        ruv = np.ctypeslib.as_array((ctypes.c_uint8 * (CH // 2 * pitch.value)).from_address(uvp.value)).reshape(
            CH // 2, pitch.value)
        recons.append((ry[:H, :W].copy(), ruv[:H // 2, :W].copy()))
    enc.h264_encoder_destroy(ctypes.c_void_p(e))
    enc.gpu_compute_destroy_image(ctypes.byref(ctx), img, mem)
    enc.bc250_gpu_destroy(ctypes.byref(ctx))
    with open(path, "wb") as f:
        f.write(stream)
    return recons


def decode(path, W, H, n):
    yuv = path + ".yuv"
    r = subprocess.run([DEC, path, yuv], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    data = np.fromfile(yuv, np.uint8)
    fs = W * H * 3 // 2
    assert data.size == n * fs, (data.size, n * fs)
    return [(data[t * fs:t * fs + W * H].reshape(H, W),
             data[t * fs + W * H:t * fs + W * H * 5 // 4].reshape(H // 2, W // 2),
             data[t * fs + W * H * 5 // 4:(t + 1) * fs].reshape(H // 2, W // 2)) for t in range(n)]


@pytest.mark.skipif(not (os.path.exists(ENC_SO) and os.path.exists(DEC)), reason="reference integration not built")
@pytest.mark.parametrize("W,H,qp,profile,slices,gop,frames", [
    (176, 144, 26, 66, 1, 4, 6),
    (176, 144, 40, 66, 2, 3, 5),
    (160, 128, 30, 77, 4, 30, 4),
    (128, 96, 22, 77, 3, 2, 4),
])
def test_reference_encoder_roundtrip_cpu(tmp_path, W, H, qp, profile, slices, gop, frames):
    path = os.path.join(str(tmp_path), "out.264")
    recons = encode_cpu(W, H, frames, qp, profile, slices, gop, path)
    dec = decode(path, W, H, frames)
    for t, ((ry, ruv), (dy, du, dv)) in enumerate(zip(recons, dec)):
        np.testing.assert_array_equal(dy, ry, err_msg=f"frame {t}: decoded luma != reconstruction")
        np.testing.assert_array_equal(du, ruv[:, 0::2], err_msg=f"frame {t}: decoded Cb != reconstruction")
        np.testing.assert_array_equal(dv, ruv[:, 1::2], err_msg=f"frame {t}: decoded Cr != reconstruction")
