"""Slice NAL units from GPU entropy coding, against the reference encoder's own.

The reference's host encoder (oracle/_ref/libh264enc_b200.so: encoder_h264.c
unchanged over this repo's gpu_compute_* boundary) encodes a sequence with
CAVLC; the same context runs with GPU entropy coding on
(b200enc_ctx_set_entropy), so each frame's slice data is also coded on the
GPU. For every frame the slice NAL units that b200enc_ctx_slice_nals
assembles - given the slice header bits the reference wrote - must be the
reference's slice NAL units byte for byte: start code, NAL header, slice
header, slice data, trailing bits and emulation prevention.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENC_SO = os.path.join(ROOT, "oracle", "_ref", "libh264enc_b200.so")


class _Bits:
    def __init__(self, data):
        self.s = "".join(f"{b:08b}" for b in data)
        self.i = 0

    def u(self, n):
        v = int(self.s[self.i:self.i + n], 2) if n else 0
        self.i += n
        return v

    def ue(self):
        z = 0
        while self.s[self.i] == "0":
            z += 1
            self.i += 1
        self.i += 1
        return (1 << z) - 1 + self.u(z)

    def se(self):
        k = self.ue()
        return (k + 1) // 2 if k & 1 else -(k // 2)


def _nal_units(stream):
    """(start, end) of each NAL unit with its 4-byte start code, in order."""
    b = bytes(stream)
    starts = []
    i = 0
    while True:
        j = b.find(b"\x00\x00\x01", i)
        if j < 0:
            break
        starts.append(j - 1 if j > 0 and b[j - 1] == 0 else j)
        i = j + 3
    return [(s, starts[k + 1] if k + 1 < len(starts) else len(b)) for k, s in enumerate(starts)]


def _rbsp(ebsp):
    out, zeros = bytearray(), 0
    for x in ebsp:
        if zeros == 2 and x == 3:
            zeros = 0
            continue
        out.append(x)
        zeros = zeros + 1 if x == 0 else 0
    return bytes(out)


def _sps(rbsp):
    r = _Bits(rbsp)
    profile = r.u(8)
    r.u(16)
    r.ue()
    if profile in (100, 110, 122, 244, 44, 83, 86, 118, 128):
        if r.ue() == 3:
            r.u(1)
        r.ue()
        r.ue()
        r.u(1)
        assert r.u(1) == 0  # no scaling matrices
    fn_bits = r.ue() + 4
    poc_type = r.ue()
    assert poc_type == 0
    return fn_bits, r.ue() + 4


def _header_bits(rbsp, idr, fn_bits, poc_bits):
    """Length in bits of the slice header the reference writes
    (encoder_h264.c:3093-3126, CAVLC)."""
    r = _Bits(rbsp)
    r.ue()
    r.ue()
    r.ue()
    r.u(fn_bits)
    if idr:
        r.ue()
    r.u(poc_bits)
    r.u(3 if not idr else 2)
    r.se()
    if r.ue() != 1:
        r.se()
        r.se()
    return r.i


@pytest.mark.parametrize("W,H,qp,slices,me", [(1280, 720, 22, 4, "full"), (1920, 1080, 30, 4, "learned_fp8"),
                                             (1920, 1080, 37, 1, "full")])
def test_gpu_slice_nals_equal_the_reference_encoders(gpu, W, H, qp, slices, me):
    from b200enc import synth
    if not os.path.exists(ENC_SO):
        pytest.skip("oracle/_ref/libh264enc_b200.so not built")
    os.environ["BC250_FORCE_QP"] = str(qp)
    os.environ["BC250_FORCE_TIER"] = "0"
    os.environ["BC250_SLICES_PER_FRAME"] = str(slices)
    os.environ["BC250_FORCE_SLICES"] = "0"
    os.environ["B200ENC_SEARCH_RANGE"] = "32"
    os.environ["B200ENC_ME"] = me
    enc = ctypes.CDLL(ENC_SO)
    L = gpu.lib()
    ctx = gpu.GpuContext()
    assert enc.bc250_gpu_init(ctypes.byref(ctx)) == 0
    assert L.b200enc_ctx_set_entropy(ctypes.byref(ctx), 1, 4) == 0
    enc.h264_encoder_create.restype = ctypes.c_void_p
    enc.h264_encoder_create.argtypes = [ctypes.POINTER(gpu.GpuContext), ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
    e = enc.h264_encoder_create(ctypes.byref(ctx), W, H, 30, 8_000_000, 66)
    assert e
    enc.h264_encoder_set_gop_size(ctypes.c_void_p(e), ctypes.c_uint32(5))
    enc.h264_encoder_encode_frame_ext.argtypes = [ctypes.c_void_p, ctypes.POINTER(gpu.GpuContext), gpu.GpuImage,
                                                  gpu.GpuMemory, ctypes.c_void_p, ctypes.c_size_t]
    img, mem = gpu.GpuImage(), gpu.GpuMemory()
    assert L.gpu_compute_create_image(ctypes.byref(ctx), W, H, 0, ctypes.byref(img), ctypes.byref(mem)) == 0
    seq = synth.Sequence(W, H, seed=qp, pan=True)
    out = np.zeros(W * H * 4, np.uint8)
    mine = np.zeros(W * H * 4, np.uint8)
    fn_bits = poc_bits = None
    try:
        for t in range(8):
            y, uv = seq.frame(t)
            assert L.gpu_compute_upload_nv12(ctypes.byref(ctx), ctypes.byref(img), mem, ctypes.c_void_p(y.ctypes.data),
                                             W, ctypes.c_void_p(uv.ctypes.data), W, W, H) == 0
            n = enc.h264_encoder_encode_frame_ext(ctypes.c_void_p(e), ctypes.byref(ctx), img, mem,
                                                  ctypes.c_void_p(out.ctypes.data), out.nbytes)
            assert n > 0
            au = out[:n].tobytes()
            want, heads, bits, ref_idc, ntype = b"", [], [], None, None
            for s0, s1 in _nal_units(au):
                hdr = au[s0 + 4]
                kind = hdr & 31
                if kind == 7:
                    fn_bits, poc_bits = _sps(_rbsp(au[s0 + 5:s1]))
                if kind not in (1, 5):
                    continue
                rb = _rbsp(au[s0 + 5:s1])
                hb = _header_bits(rb, kind == 5, fn_bits, poc_bits)
                head = int("".join(f"{x:08b}" for x in rb)[:hb], 2)
                heads.append(np.frombuffer((head << (128 - hb)).to_bytes(16, "big"), np.uint8))
                bits.append(hb)
                ref_idc, ntype = hdr >> 5, kind
                want += au[s0:s1]
            assert len(heads) == slices
            slot = L.gpu_compute_submitted_slot(ctypes.byref(ctx))
            h = np.ascontiguousarray(np.stack(heads))
            hb = np.array(bits, np.int32)
            written = ctypes.c_size_t()
            assert L.b200enc_ctx_slice_nals(ctypes.byref(ctx), slot, ctypes.c_void_p(h.ctypes.data),
                                            ctypes.c_void_p(hb.ctypes.data), ref_idc, ntype,
                                            ctypes.c_void_p(mine.ctypes.data), mine.nbytes,
                                            ctypes.byref(written)) == 0
            got = mine[:written.value].tobytes()
            assert got == want, f"frame {t}: {len(got)} vs {len(want)} bytes"
    finally:
        enc.h264_encoder_destroy(ctypes.c_void_p(e))
        L.gpu_compute_destroy_image(ctypes.byref(ctx), img, mem)
        L.bc250_gpu_destroy(ctypes.byref(ctx))
