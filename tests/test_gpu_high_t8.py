"""A High-profile stream with 8x8-transform P macroblocks, made on the GPU and
decoded by the reference's decoder.

Every stage runs on the GPU through the C-ABI: full search, the P chain with
the 8x8 luma transform (b200enc_p_frame_t8; for every macroblock, or chosen
per macroblock with the flags passed on), the I16x16 wavefront, tile
deblocking with 8x8-transform macroblocks, and CAVLC slices with
transform_size_8x8_flag and the four interleaved 4x4 blocks of each 8x8
block (b200enc_cavlc_slices, transform8x8). The parameter sets (High profile,
transform_8x8_mode_flag), slice headers and NAL framing are written here. The
reference's H.264 decoder (oracle/_ref/h264dec, its CAVLC 8x8 path,
h264_mb_cavlc.c:134-180, and h264d_idct8_add) must reconstruct every frame
exactly as the GPU did - which pins the 8x8 P chain's reconstruction, the
entropy coding of 8x8 blocks and the deblocking of 8x8 macroblocks together.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEC = os.path.join(ROOT, "oracle", "_ref", "h264dec")


class _Bits:
    def __init__(self):
        self.b = []

    def u(self, n, v):
        self.b.append(format(v, f"0{n}b") if n else "")

    def ue(self, v):
        c = v + 1
        self.b.append("0" * (c.bit_length() - 1) + format(c, "b"))

    def se(self, v):
        self.ue(2 * v - 1 if v > 0 else -2 * v)

    def rbsp(self):
        s = "".join(self.b) + "1"
        s += "0" * (-len(s) % 8)
        return bytes(int(s[i:i + 8], 2) for i in range(0, len(s), 8))

    def value(self):
        s = "".join(self.b)
        return int(s, 2) if s else 0, len(s)


def _nal(ref_idc, kind, rbsp):
    out, zeros = bytearray(), 0
    for x in rbsp:
        if zeros == 2 and x <= 3:
            out.append(3)
            zeros = 0
        out.append(x)
        zeros = zeros + 1 if x == 0 else 0
    return b"\x00\x00\x00\x01" + bytes([(ref_idc << 5) | kind]) + bytes(out)


def _sps(mbw, mbh, crop_bottom=0):
    b = _Bits()
    b.u(8, 100)          # profile_idc: High
    b.u(8, 0)
    b.u(8, 40)
    b.ue(0)              # seq_parameter_set_id
    b.ue(1)              # chroma_format_idc 4:2:0
    b.ue(0)
    b.ue(0)
    b.u(1, 0)
    b.u(1, 0)            # no scaling matrices
    b.ue(4)              # log2_max_frame_num - 4
    b.ue(0)              # pic_order_cnt_type
    b.ue(4)              # log2_max_pic_order_cnt_lsb - 4
    b.ue(1)
    b.u(1, 0)
    b.ue(mbw - 1)
    b.ue(mbh - 1)
    b.u(1, 1)            # frame_mbs_only
    b.u(1, 1)            # direct_8x8_inference
    b.u(1, int(crop_bottom > 0))
    if crop_bottom:      # frame cropping, in units of two luma rows (4:2:0 frames)
        b.ue(0)
        b.ue(0)
        b.ue(0)
        b.ue(crop_bottom // 2)
    b.u(1, 0)
    return _nal(3, 7, b.rbsp())


def _pps(qp, t8=True):
    b = _Bits()
    b.ue(0)
    b.ue(0)
    b.u(1, 0)            # CAVLC
    b.u(1, 0)
    b.ue(0)
    b.ue(0)
    b.ue(0)
    b.u(1, 0)
    b.u(2, 0)
    b.se(qp - 26)
    b.se(0)
    b.se(0)
    b.u(1, 1)            # deblocking_filter_control_present
    b.u(1, 0)
    b.u(1, 0)
    b.u(1, int(t8))      # transform_8x8_mode_flag
    b.u(1, 0)
    b.se(0)
    return _nal(3, 8, b.rbsp())


def _slice_header(first_mb, idr, frame_num):
    b = _Bits()
    b.ue(first_mb)
    b.ue(7 if idr else 5)
    b.ue(0)
    b.u(8, frame_num & 255)
    if idr:
        b.ue(0)
    b.u(8, (2 * frame_num) & 255)
    if not idr:
        b.u(1, 0)
        b.u(1, 0)
        b.u(1, 0)
    else:
        b.u(1, 0)
        b.u(1, 0)
    b.se(0)
    b.ue(0)
    b.se(0)
    b.se(0)
    return b.value()


def _i420(nv12_y, nv12_uv, W, H):
    return nv12_y[:H, :W], nv12_uv[:H // 2, 0:W:2], nv12_uv[:H // 2, 1:W:2]


def encode_high(gpu, seq, W, H, qp, ns, n, t8, rng=16):
    """Encodes n frames of `seq` (IDR, then P frames) on the GPU with the 8x8
    luma transform mode t8 (0: 4x4 only and no transform_8x8_mode_flag, 1:
    every macroblock, 2: chosen per macroblock). Returns the Annex B NAL units
    (SPS, PPS, then each frame's slices), the deblocked reconstructions (I420
    planes at W x H) and per-P-frame counts (coded 8x8, 8x8, 4x4
    macroblocks)."""
    import torch
    L = gpu.lib()
    CW, CH = gpu.coded(W, H)
    mbw, mbh = CW // 16, CH // 16
    mbs = mbw * mbh
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    nals = [_sps(mbw, mbh, CH - H), _pps(qp, t8 != 0)]
    recons, ref, counts = [], None, []
    flags = torch.ones(mbs, dtype=torch.uint8, device="cuda")
    for t in range(n):
        cur = gpu.NV12.from_host(*seq.frame(t))
        out = gpu.Outputs(W, H)
        rec = gpu.NV12(W, H)
        idr = t == 0
        if idr:
            scr = gpu.scratch(mbh)
            gpu.i_frame(cur, W, H, CW, CH, qp, ns, out, rec, scr)
        else:
            gpu.me_full_search(cur, ref, W, H, CW, CH, rng, 5, 512, out.mv)
            flags.fill_(7)
            gpu.p_frame_t8(cur, ref, W, H, CW, CH, qp, out.mv, out, rec, t8, flags)
        recd = gpu.NV12(W, H)
        st = torch.zeros(4, dtype=torch.int32, device="cuda")
        assert L.b200enc_deblock_tiles_t8(mbw, mbh, qp, int(idr), vp(out.nz), None if idr else vp(flags),
                                          vp(out.mv), rec.yp(), rec.uvp(), recd.yp(), recd.uvp(), rec.pitch,
                                          vp(st), None) == 0
        heads = [_slice_header(s * mbs // ns, idr, t) for s in range(ns)]
        slices = gpu.cavlc_slices(mbw, mbh, qp, int(idr), ns, out.levels.data_ptr(), out.dc.data_ptr(),
                                  out.nz.data_ptr(), out.pred_mode.data_ptr(), out.mv.data_ptr(), headers=heads,
                                  transform8x8=0 if idr or t8 == 0 else 1,
                                  t8_flags=None if idr or t8 == 0 else flags.data_ptr())
        nals += [_nal(3 if idr else 2, 5 if idr else 1, s) for s in slices]
        torch.cuda.synchronize()
        assert st.cpu().tolist()[:2] == [0, 0]
        if not idr:
            f8 = flags.cpu().numpy()
            assert set(np.unique(f8)) <= {0, 1}
            coded = (out.nz[:, :16].cpu().numpy() != 0).any(axis=1)
            counts.append((int((coded & (f8 == 1)).sum()), int((f8 == 1).sum()), int((f8 == 0).sum())))
        recons.append(_i420(recd.y.cpu().numpy(), recd.uv.cpu().numpy(), W, H))
        ref = recd
    return nals, recons, counts


def decode(path, W, H, n):
    yuv = path + ".yuv"
    r = subprocess.run([DEC, path, yuv], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    data = np.fromfile(yuv, np.uint8)
    fs = W * H * 3 // 2
    assert data.size == n * fs, (data.size, n * fs)
    return [(f[:W * H].reshape(H, W), f[W * H:W * H * 5 // 4].reshape(H // 2, W // 2),
             f[W * H * 5 // 4:].reshape(H // 2, W // 2)) for f in (data[t * fs:(t + 1) * fs] for t in range(n))]


@pytest.mark.skipif(not os.path.exists(DEC), reason="oracle/_ref/h264dec not built")
@pytest.mark.parametrize("W,H,qp,ns,n", [(640, 352, 26, 2, 6), (1280, 720, 33, 4, 5), (320, 192, 18, 1, 5)])
@pytest.mark.parametrize("t8", [1, 2])
def test_high_profile_8x8_stream_decodes_to_the_gpu_reconstruction(gpu, tmp_path, W, H, qp, ns, n, t8):
    from b200enc import synth
    seq = synth.Sequence(W, H, seed=qp, pan=True)
    nals, recons, counts = encode_high(gpu, seq, W, H, qp, ns, n, t8)
    assert sum(c[0] for c in counts) > 0  # the P frames did code 8x8 luma blocks
    n8, n4 = sum(c[1] for c in counts), sum(c[2] for c in counts)
    if t8 == 1:
        assert n4 == 0
    else:  # the per-macroblock choice took both sizes
        assert n8 > 0 and n4 > 0, (n8, n4)
    path = os.path.join(str(tmp_path), "high8x8.264")
    with open(path, "wb") as f:
        f.write(b"".join(nals))
    for t, (got, want) in enumerate(zip(decode(path, W, H, n), recons)):
        for plane, a, b in zip("YUV", got, want):
            np.testing.assert_array_equal(a, b, err_msg=f"frame {t} {plane}")


@pytest.mark.skipif(not os.path.exists(DEC), reason="oracle/_ref/h264dec not built")
@pytest.mark.parametrize("qp", [22, 27, 32, 37])
def test_high_profile_1080p_r32_qp_sweep(gpu, tmp_path, qp):
    """The High configuration: 1920x1080 IPPP, full search +-32, 4x4 and 8x8
    transforms chosen per macroblock, deblocking, on the seeded 1080p
    generator (pan, noise patch); the reference decoder reconstructs every
    frame exactly as the GPU did."""
    from b200enc import synth
    W, H, n = 1920, 1080, 6
    seq = synth.workload("h264_1080p", seed=0, stream=qp)
    nals, recons, counts = encode_high(gpu, seq, W, H, qp, 1, n, 2, rng=32)
    assert sum(c[1] for c in counts) > 0 and sum(c[2] for c in counts) > 0
    path = os.path.join(str(tmp_path), "high1080.264")
    with open(path, "wb") as f:
        f.write(b"".join(nals))
    for t, (got, want) in enumerate(zip(decode(path, W, H, n), recons)):
        for plane, a, b in zip("YUV", got, want):
            np.testing.assert_array_equal(a, b, err_msg=f"frame {t} {plane}")
