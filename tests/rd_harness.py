"""Rate-distortion measurement through the reference's own host encoder.
TEST INFRASTRUCTURE: used by tests/test_gpu_bdrate.py and tests/rd_report.py.

The reference's encoder_h264.c (unchanged, in oracle/_ref/libh264enc_b200.so)
drives libb200enc.so through the gpu_compute_* boundary and writes the
bitstream; the bits are the stream's size, the distortion is the PSNR of the
reconstruction the GPU kept (which the round-trip tests prove equal to the
reference decoder's output). The motion-estimation form of P frames is set
on the context with b200enc_ctx_set_me.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENC_SO = os.path.join(ROOT, "oracle", "_ref", "libh264enc_b200.so")

PLAIN, LEARNED, CANDIDATES, LEARNED_FP8 = 0, 1, 2, 3


def available():
    return os.path.exists(ENC_SO)


def make_frames(W, H, n, seed=0):
    from b200enc import synth
    seq = synth.Sequence(W, H, seed=seed, pan=True, noise_patch=True)
    return [seq.frame(t) for t in range(n)]


def encode(gpu, frames, W, H, qp, me_mode, conf=0.9, weights=None, profile=77, gop=60, search_range=32):
    """Encodes `frames` at fixed QP; returns dict(bits, psnr_y, psnr_yuv,
    frame_bits, learned, fallback, early)."""
    from b200enc import rd
    os.environ["BC250_FORCE_QP"] = str(qp)
    os.environ["BC250_FORCE_TIER"] = "0"
    os.environ["BC250_SLICES_PER_FRAME"] = "1"
    os.environ["BC250_FORCE_SLICES"] = "0"
    os.environ["B200ENC_SEARCH_RANGE"] = str(search_range)
    enc = ctypes.CDLL(ENC_SO)
    L = gpu.lib()
    ctx = gpu.GpuContext()
    assert enc.bc250_gpu_init(ctypes.byref(ctx)) == 0
    rc = L.b200enc_ctx_set_me(ctypes.byref(ctx), me_mode, weights.encode() if weights else None, ctypes.c_float(conf))
    assert rc == 0, f"b200enc_ctx_set_me rc={rc}"
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
    out = np.zeros(W * H * 4, np.uint8)
    frame_bits, psnr_y, psnr_yuv = [], [], []
    learned = fallback = early = 0
    CH = (H + 15) // 16 * 16
    for t, (y, uv) in enumerate(frames):
        assert L.gpu_compute_upload_nv12(ctypes.byref(ctx), ctypes.byref(img), mem, ctypes.c_void_p(y.ctypes.data), W,
                                         ctypes.c_void_p(uv.ctypes.data), W, W, H) == 0
        n = enc.h264_encoder_encode_frame_ext(ctypes.c_void_p(e), ctypes.byref(ctx), img, mem,
                                              ctypes.c_void_p(out.ctypes.data), out.nbytes)
        assert n > 0, f"frame {t}: encoder returned {n}"
        frame_bits.append(8 * n)
        yp, uvp, pitch = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int()
        assert L.b200enc_ctx_recon(ctypes.byref(ctx), ctypes.byref(yp), ctypes.byref(uvp), ctypes.byref(pitch)) == 0
        ry = gpu.device_view(yp.value, CH * pitch.value).cpu().numpy().reshape(CH, pitch.value)[:H, :W]
        ruv = gpu.device_view(uvp.value, CH // 2 * pitch.value).cpu().numpy().reshape(CH // 2, pitch.value)
        ruv = ruv[:H // 2, :W]
        py, _, _, pyuv = rd.psnr_yuv(y, uv, ry, ruv)
        psnr_y.append(py)
        psnr_yuv.append(pyuv)
        if me_mode != PLAIN and t > 0:
            li, fb, ea = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            assert L.b200enc_ctx_me_stats(ctypes.byref(ctx), ctypes.byref(li), ctypes.byref(fb), ctypes.byref(ea)) == 0
            learned += li.value
            fallback += fb.value
            early += ea.value
    enc.h264_encoder_destroy(ctypes.c_void_p(e))
    L.gpu_compute_destroy_image(ctypes.byref(ctx), img, mem)
    L.bc250_gpu_destroy(ctypes.byref(ctx))
    return dict(bits=int(sum(frame_bits)), psnr_y=float(np.mean(psnr_y)), psnr_yuv=float(np.mean(psnr_yuv)),
                frame_bits=frame_bits, learned=learned, fallback=fallback, early=early)


def rd_curves(gpu, frames, W, H, modes, qps=(22, 27, 32, 37), conf=0.9, weights=None, profile=77):
    """{mode: [encode() result per QP]}"""
    return {m: [encode(gpu, frames, W, H, qp, m, conf, weights, profile) for qp in qps] for m in modes}


def bd_rate(anchor, test, key="psnr_yuv"):
    from b200enc import rd
    return rd.bd_rate([r["bits"] for r in anchor], [r[key] for r in anchor], [r["bits"] for r in test],
                      [r[key] for r in test])
