"""Encode -> decode round trip through the reference's own host encoder.

The reference's encoder_h264.c (unchanged, compiled against this repo's
include/gpu_compute.h into oracle/_ref/libh264enc_b200.so by
oracle/Makefile) drives libb200enc.so through the gpu_compute_* boundary:
the B200 kernels produce the levels, DC, modes, MVs and nonzero masks, the
reference host code writes CAVLC or CABAC slices. The stream is decoded by
the reference's own H.264 decoder (oracle/_ref/h264dec), and every decoded
frame must equal the reconstruction the GPU kept as its reference, bit for
bit: that is what makes the GPU's reconstruction (spec deblocking included)
a valid reference picture.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENC_SO = os.path.join(ROOT, "oracle", "_ref", "libh264enc_b200.so")
DEC = os.path.join(ROOT, "oracle", "_ref", "h264dec")


def _encode(gpu, W, H, frames, qp, profile, slices, gop, tmp_path, seed=3, search_range=16, me="full", seq=None):
    from b200enc import synth
    os.environ["BC250_FORCE_QP"] = str(qp)
    os.environ["BC250_FORCE_TIER"] = "0"
    os.environ["BC250_SLICES_PER_FRAME"] = str(slices)
    os.environ["BC250_FORCE_SLICES"] = "0"
    os.environ["B200ENC_SEARCH_RANGE"] = str(search_range)  # read by bc250_gpu_init
    os.environ["B200ENC_ME"] = me
    enc = ctypes.CDLL(ENC_SO)
    L = gpu.lib()
    ctx = gpu.GpuContext()
    assert enc.bc250_gpu_init(ctypes.byref(ctx)) == 0
    enc.h264_encoder_create.restype = ctypes.c_void_p
    enc.h264_encoder_create.argtypes = [ctypes.POINTER(gpu.GpuContext), ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
    e = enc.h264_encoder_create(ctypes.byref(ctx), W, H, 30, 8_000_000, profile)
    assert e
    enc.h264_encoder_set_gop_size(ctypes.c_void_p(e), ctypes.c_uint32(gop))
    enc.h264_encoder_encode_frame_ext.argtypes = [ctypes.c_void_p, ctypes.POINTER(gpu.GpuContext), gpu.GpuImage,
                                                  gpu.GpuMemory, ctypes.c_void_p, ctypes.c_size_t]
    img, mem = gpu.GpuImage(), gpu.GpuMemory()
    assert L.gpu_compute_create_image(ctypes.byref(ctx), W, H, 0, ctypes.byref(img), ctypes.byref(mem)) == 0
    if seq is None:
        seq = synth.Sequence(W, H, seed=seed, pan=True)
    out = np.zeros(W * H * 4, np.uint8)
    stream, recons = bytearray(), []
    for t in range(frames):
        y, uv = seq.frame(t)
        assert L.gpu_compute_upload_nv12(ctypes.byref(ctx), ctypes.byref(img), mem, ctypes.c_void_p(y.ctypes.data), W,
                                         ctypes.c_void_p(uv.ctypes.data), W, W, H) == 0
        n = enc.h264_encoder_encode_frame_ext(ctypes.c_void_p(e), ctypes.byref(ctx), img, mem,
                                              ctypes.c_void_p(out.ctypes.data), out.nbytes)
        assert n > 0, f"frame {t}: encoder returned {n}"
        stream += out[:n].tobytes()
        yp, uvp, pitch = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int()
        assert L.b200enc_ctx_recon(ctypes.byref(ctx), ctypes.byref(yp), ctypes.byref(uvp), ctypes.byref(pitch)) == 0
        CH = (H + 15) // 16 * 16
        ry = gpu.device_view(yp.value, CH * pitch.value).cpu().numpy().reshape(CH, pitch.value)
        ruv = gpu.device_view(uvp.value, CH // 2 * pitch.value).cpu().numpy().reshape(CH // 2, pitch.value)
        recons.append((ry[:H, :W].copy(), ruv[:H // 2, :W].copy()))
    enc.h264_encoder_destroy(ctypes.c_void_p(e))
    L.gpu_compute_destroy_image(ctypes.byref(ctx), img, mem)
    L.bc250_gpu_destroy(ctypes.byref(ctx))
    path = os.path.join(str(tmp_path), "out.264")
    with open(path, "wb") as f:
        f.write(stream)
    return path, recons


def _decode(path, W, H, n):
    yuv = path + ".yuv"
    r = subprocess.run([DEC, path, yuv], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    data = np.fromfile(yuv, np.uint8)
    fs = W * H * 3 // 2
    assert data.size == n * fs, (data.size, n * fs)
    frames = []
    for t in range(n):
        f = data[t * fs:(t + 1) * fs]
        frames.append((f[:W * H].reshape(H, W), f[W * H:W * H * 5 // 4].reshape(H // 2, W // 2),
                       f[W * H * 5 // 4:].reshape(H // 2, W // 2)))
    return frames


@pytest.mark.skipif(not (os.path.exists(ENC_SO) and os.path.exists(DEC)), reason="reference integration not built")
@pytest.mark.parametrize("W,H,qp,profile,slices,gop,frames", [
    (320, 240, 26, 66, 1, 8, 10),     # Baseline (CAVLC), one IDR refresh
    (640, 480, 30, 66, 4, 30, 6),     # 4 slices
    (640, 480, 22, 77, 1, 30, 6),     # Main (CABAC)
    (176, 144, 40, 66, 2, 3, 7),      # high QP, frequent IDR
    (1280, 720, 27, 77, 4, 60, 4),
])
def test_reference_encoder_roundtrip(gpu, tmp_path, W, H, qp, profile, slices, gop, frames):
    path, recons = _encode(gpu, W, H, frames, qp, profile, slices, gop, tmp_path)
    dec = _decode(path, W, H, frames)
    for t, ((ry, ruv), (dy, du, dv)) in enumerate(zip(recons, dec)):
        np.testing.assert_array_equal(dy, ry, err_msg=f"frame {t}: decoded luma != GPU reconstruction")
        np.testing.assert_array_equal(du, ruv[:, 0::2], err_msg=f"frame {t}: decoded Cb != GPU reconstruction")
        np.testing.assert_array_equal(dv, ruv[:, 1::2], err_msg=f"frame {t}: decoded Cr != GPU reconstruction")


@pytest.mark.skipif(not (os.path.exists(ENC_SO) and os.path.exists(DEC)), reason="reference integration not built")
@pytest.mark.parametrize("qp,profile,me", [
    (27, 66, "full"),          # Baseline (CAVLC), the bench's QP
    (27, 77, "full"),          # Main (CABAC)
    (22, 77, "learned_fp8"),   # the learned form (network in FP8), CABAC
    (37, 66, "learned_fp8"),   # the learned form, CAVLC, coarse QP
])
def test_reference_encoder_roundtrip_1080p_r32(gpu, tmp_path, qp, profile, me):
    """1920x1080 at the bench's search range 32 on the bench's generator:
    the reference host encoder's stream, decoded by the reference decoder,
    equals the GPU's reconstruction in every frame (I plus 7 P frames, the
    learned form's candidates taking over from the third frame)."""
    from b200enc import synth
    W, H, n = 1920, 1080, 8
    seq = synth.workload("h264_1080p", seed=0, stream=qp)
    try:
        path, recons = _encode(gpu, W, H, n, qp, profile, 1, 60, tmp_path, search_range=32, me=me, seq=seq)
    finally:
        os.environ.pop("B200ENC_ME", None)
        os.environ.pop("B200ENC_SEARCH_RANGE", None)
    dec = _decode(path, W, H, n)
    for t, ((ry, ruv), (dy, du, dv)) in enumerate(zip(recons, dec)):
        np.testing.assert_array_equal(dy, ry, err_msg=f"frame {t}: decoded luma != GPU reconstruction")
        np.testing.assert_array_equal(du, ruv[:, 0::2], err_msg=f"frame {t}: decoded Cb != GPU reconstruction")
        np.testing.assert_array_equal(dv, ruv[:, 1::2], err_msg=f"frame {t}: decoded Cr != GPU reconstruction")
