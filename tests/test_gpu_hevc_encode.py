"""The reference's host HEVC encoder with its motion search's half-sample
planes built on the GPU (bc250-vaapi_b200/binding/hevc_hpel_binding.c,
compiled with the unchanged encoder_h265.c into
oracle/_ref/libhevcenc_b200.so) writes byte for byte the stream of the
unchanged reference encoder (oracle/_ref/libhevcref.so) on the same frames,
at 8 bits (1920x1080, wavefront parallel rows, several QPs) and at 10 bits
(Main10, P010 input), every P picture's planes having come from the GPU; and
the reference's own decoder tool (oracle/_ref/hevcps) decodes the stream."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libhevcref.so")
GPU_SO = os.path.join(ROOT, "oracle", "_ref", "libhevcenc_b200.so")
HEVCPS = os.path.join(ROOT, "oracle", "_ref", "hevcps")
needs = pytest.mark.skipif(not (os.path.exists(REF_SO) and os.path.exists(GPU_SO)), reason="HEVC builds missing")


def frames_8bit(W, H, n, seed):
    from b200enc import synth
    seq = synth.Sequence(W, H, seed=seed, pan=True, noise_patch=W >= 1280)
    return [seq.frame(t) for t in range(n)]


def frames_p010(W, H, n, seed):
    """P010: 10-bit samples 64..940 (sigma-12 grain) in the top ten bits of 16-bit words."""
    rs = np.random.Generator(np.random.PCG64(seed))
    out = []
    for y8, uv8 in frames_8bit(W, H, n, seed):
        y = np.clip(np.rint(64 + y8 * (876 / 255) + rs.normal(0, 12, y8.shape)), 64, 940).astype(np.uint16)
        uv = np.clip(np.rint(64 + uv8 * (876 / 255)), 64, 940).astype(np.uint16)
        out.append((y << 6, uv << 6))
    return out


def encode(so, frames, W, H, bit_depth, qp, threads=8):
    os.environ["BC250_HEVC_QP"] = str(qp)
    os.environ["BC250_HEVC_THREADS"] = str(threads)
    try:
        L = ctypes.CDLL(so)
        L.hevc_encoder_create_depth.restype = ctypes.c_void_p
        L.hevc_encoder_create_depth.argtypes = [ctypes.c_void_p] + [ctypes.c_uint32] * 4 + [ctypes.c_int]
        L.hevc_encoder_set_gop_size.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.hevc_encoder_encode_raw.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
        L.hevc_encoder_destroy.argtypes = [ctypes.c_void_p]
        e = L.hevc_encoder_create_depth(None, W, H, 30, 8_000_000, bit_depth)
        assert e
        L.hevc_encoder_set_gop_size(e, 60)
        out = np.zeros(W * H * 6, np.uint8)
        stream = bytearray()
        for y, uv in frames:
            n = L.hevc_encoder_encode_raw(e, y.ctypes.data, y.strides[0], uv.ctypes.data, uv.strides[0],
                                          out.ctypes.data, out.nbytes)
            assert n > 0, n
            stream += out[:n].tobytes()
        L.hevc_encoder_destroy(e)
        return bytes(stream), L
    finally:
        os.environ.pop("BC250_HEVC_QP", None)
        os.environ.pop("BC250_HEVC_THREADS", None)


def gpu_stats(L):
    a, b = ctypes.c_long(), ctypes.c_long()
    L.b200_hevc_hpel_stats(ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


@needs
@pytest.mark.parametrize("W,H,bit_depth,qp,n", [(1920, 1080, 8, 22, 6), (1920, 1080, 8, 32, 6), (1280, 720, 8, 37, 8),
                                               (416, 240, 10, 27, 8), (1920, 1080, 10, 30, 4)])
def test_gpu_planes_give_the_reference_stream(gpu, tmp_path, W, H, bit_depth, qp, n):
    frames = frames_8bit(W, H, n, seed=W + qp) if bit_depth == 8 else frames_p010(W, H, n, seed=W + qp)
    want, _ = encode(REF_SO, frames, W, H, bit_depth, qp)
    g0 = None
    got, L = encode(GPU_SO, frames, W, H, bit_depth, qp)
    pics, failed = gpu_stats(L)
    assert failed == 0
    assert pics >= n - 1, f"only {pics} of {n - 1} P pictures built their planes on the GPU"
    assert got == want, f"streams differ ({len(got)} vs {len(want)} bytes)"
    if os.path.exists(HEVCPS):
        path = os.path.join(str(tmp_path), "s.265")
        with open(path, "wb") as f:
            f.write(got)
        r = subprocess.run([HEVCPS, "-q", path, path + ".yuv"], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        assert os.path.getsize(path + ".yuv") > 0
