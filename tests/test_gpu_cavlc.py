"""GPU CAVLC (b200enc_cavlc_slices) against the reference's own CAVLC writer.

The oracle here is the reference host encoder itself: oracle/cavlc_shim.c
includes its encoder_h264.c and runs its macroblock loop and encoders over
the same staged outputs (oracle/_ref/libcavlcref.so). Every slice's bytes must
be identical: on synthetic outputs built to reach every table (dense and
sparse blocks, trailing ones, level escapes, long zero runs, skip runs, all
four nC classes, every intra mode at slice and picture edges), with and
without slice headers in front, and on the outputs of real 1080p encodes
(I and P frames, plain and learned forms, several QPs and slice counts).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(oracle_mod):
    if not oracle_mod.cavlc_ref_available():
        pytest.skip("oracle/_ref/libcavlcref.so not built")
    return oracle_mod


def _synthetic(rs, mbw, mbh, intra):
    mbs = mbw * mbh
    levels = np.zeros((mbs, 24, 16), np.int16)
    dc = np.zeros((mbs, 24), np.int32)
    mv = np.zeros((mbs, 4), np.int32)
    for mb in range(mbs):
        kind = rs.random()
        if not intra and kind < 0.3:
            continue  # a skip candidate: nothing coded, zero vector
        dens = rs.choice([0.05, 0.2, 0.6, 1.0])
        big = rs.random() < 0.15
        for b in range(24):
            if rs.random() < 0.35:
                continue
            m = rs.random(16) < dens
            v = rs.choice([-1, 1], 16) * np.where(rs.random(16) < 0.6, 1, rs.integers(2, 12, 16))
            if big:
                v = np.where(rs.random(16) < 0.3, rs.integers(-3000, 3001, 16), v)
            levels[mb, b] = np.where(m, v, 0).astype(np.int16)
        dc[mb, :16] = rs.integers(-4000, 4001, 16) * (rs.random(16) < 0.5)
        dc[mb, 16:] = rs.integers(-900, 901, 8) * (rs.random(8) < 0.6)
        mv[mb, :2] = rs.integers(-40, 41, 2) * (rs.random() < 0.8)
    nz = np.zeros((mbs, 24), np.uint32)
    for p in range(16):
        nz |= (levels[:, :, p] != 0).astype(np.uint32) << p
    pm = rs.integers(0, 16, mbs).astype(np.uint32)
    return levels, dc, nz, pm, mv


def _gpu_slices(gpu, mbw, mbh, qp, intra, ns, levels, dc, nz, pm, mv, headers=None, quality=4):
    import torch
    t = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (levels, dc, nz.view(np.int32), pm.view(np.int32), mv)]
    return gpu.cavlc_slices(mbw, mbh, qp, intra, ns, *[x.data_ptr() for x in t], headers=headers,
                            quality_level=quality)


def _ref_slices(ref, mbw, mbh, qp, intra, ns, levels, dc, nz, pm, mv, quality=4):
    mbs = mbw * mbh
    return [ref.ref_cavlc_slice_data(mbw, mbh, qp, intra, s * mbs // ns, (s + 1) * mbs // ns, levels, dc, nz, pm, mv,
                                     quality_level=quality) for s in range(ns)]


def _bits(b):
    return "".join(f"{x:08b}" for x in b)


@pytest.mark.parametrize("intra", [1, 0])
@pytest.mark.parametrize("mbw,mbh,ns", [(1, 1, 1), (11, 9, 1), (11, 9, 3), (30, 17, 4), (7, 23, 16)])
@pytest.mark.parametrize("qp", [12, 27, 45])
def test_synthetic_slices_match_reference(gpu, ref, intra, mbw, mbh, ns, qp):
    rs = np.random.Generator(np.random.PCG64(mbw * 131 + mbh * 7 + ns * 3 + qp + intra))
    args = _synthetic(rs, mbw, mbh, intra)
    got = _gpu_slices(gpu, mbw, mbh, qp, intra, ns, *args)
    want = _ref_slices(ref, mbw, mbh, qp, intra, ns, *args)
    for s, (g, w) in enumerate(zip(got, want)):
        assert g == w, f"slice {s}: {len(g)} vs {len(w)} bytes, first difference at byte " \
                       f"{next((i for i in range(min(len(g), len(w))) if g[i] != w[i]), min(len(g), len(w)))}"


@pytest.mark.parametrize("quality", [4, 5])
def test_skip_rule_follows_quality_level(gpu, ref, quality):
    rs = np.random.Generator(np.random.PCG64(99 + quality))
    mbw, mbh = 13, 8
    levels, dc, nz, pm, mv = _synthetic(rs, mbw, mbh, 0)
    # macroblocks with no luma levels and tiny chroma DC terms, where the rule differs
    for mb in range(0, mbw * mbh, 3):
        levels[mb] = 0
        nz[mb] = 0
        dc[mb] = 0
        dc[mb, 16:20] = rs.integers(-1, 2, 4)
        mv[mb, :2] = 0
    got = _gpu_slices(gpu, mbw, mbh, 30, 0, 2, levels, dc, nz, pm, mv, quality=quality)
    want = _ref_slices(ref, mbw, mbh, 30, 0, 2, levels, dc, nz, pm, mv, quality=quality)
    assert got == want


def test_headers_precede_the_slice_data(gpu, ref):
    rs = np.random.Generator(np.random.PCG64(5))
    mbw, mbh, ns = 12, 7, 3
    args = _synthetic(rs, mbw, mbh, 0)
    heads = [(int.from_bytes(rs.bytes(16), "big") >> (128 - n), n) for n in (1, 37, 128)]
    got = _gpu_slices(gpu, mbw, mbh, 33, 0, ns, *args, headers=heads)
    want = _ref_slices(ref, mbw, mbh, 33, 0, ns, *args)
    for (bits, n), g, w in zip(heads, got, want):
        data = _bits(w).rstrip("0")[:-1]  # the reference's slice data without its trailing bits
        exp = (format(bits, f"0{n}b") if n else "") + data + "1"
        exp += "0" * (-len(exp) % 8)
        assert _bits(g) == exp


def _encode_outputs(gpu, W, H, qp, ns, me_mode, n, seed):
    """Device outputs of n frames (I then P) of the synthetic workload through
    an encoding context; yields (intra, device pointers, host copies)."""
    import torch
    from b200enc import synth
    seq = synth.workload("h264_1080p", seed=seed, stream=3)
    ctx = gpu.Context()
    ctx.configure(search_range=32, lam=5, zero_thresh=512, coded_clamp=True, deblock=1)
    ctx.set_me(me_mode)
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    try:
        for t in range(n):
            fr = gpu.NV12.from_host(*seq.frame(t))
            ctx.encode_device(fr, W, H, qp, t == 0, ns, False)
            ptrs = [ctypes.c_void_p() for _ in range(5)]
            assert ctx.L.b200enc_ctx_device_outputs(ctypes.byref(ctx.ctx), *[ctypes.byref(p) for p in ptrs]) == 0
            torch.cuda.synchronize()
            sizes = [mbs * 768, mbs * 96, mbs * 96, mbs * 4, mbs * 16]
            host = [gpu.device_view(p.value, z).cpu().numpy() for p, z in zip(ptrs, sizes)]
            host = [host[0].view(np.int16).reshape(mbs, 24, 16), host[1].view(np.int32).reshape(mbs, 24),
                    host[2].view(np.uint32).reshape(mbs, 24), host[3].view(np.uint32), host[4].view(np.int32).reshape(mbs, 4)]
            yield t == 0, [p.value for p in ptrs], host
    finally:
        ctx.close()


@pytest.mark.parametrize("qp,ns,me_mode", [(22, 4, 0), (27, 4, 3), (37, 1, 0), (32, 8, 3)])
def test_encoded_1080p_frames_match_reference(gpu, ref, qp, ns, me_mode):
    W, H = 1920, 1080
    mbw, mbh = 120, 68
    for intra, dev, host in _encode_outputs(gpu, W, H, qp, ns, me_mode, 4, seed=qp):
        got = gpu.cavlc_slices(mbw, mbh, qp, intra, ns, *dev)
        want = _ref_slices(ref, mbw, mbh, qp, int(intra), ns, *host)
        assert got == want, f"intra={intra}"
