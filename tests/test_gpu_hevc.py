"""HEVC primitives (csrc/hevc.cu) against the reference's own compiled
routines (oracle/_ref/libhevcref.so: hevc_intra.c linked as is, and the HEVC
encoder's static build_hpel exposed by oracle/hevc_shim.c), bit for bit:

* 4x4 DCT-II / DST-VII transform + quant and dequant + inverse at 8 and 10
  bits, 8x8 at 8 and 10 bits, over QPs 0..63 (including out-of-range QPs the
  reference clamps), every rounding offset class, zero blocks, and extreme
  inputs that drive the int16 saturation of both transform passes;
* the motion search's whole- and half-sample planes (margin 16) on frames
  from 16x16 to 1920x1088;
* the 8x8 CU motion search (starting points, downhill walk, half/quarter
  refinement, MVD-bit cost): vector, predictor index, cost and SAD of every
  CU of a frame;
* the intra 4x4 luma mode choice (mode and prediction) of PUs across picture
  edges, z-order availability and slice starts.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEVC_SO = os.path.join(ROOT, "oracle", "_ref", "libhevcref.so")
needs_ref = pytest.mark.skipif(not os.path.exists(HEVC_SO), reason="reference HEVC routines not built")


def _ref():
    L = ctypes.CDLL(HEVC_SO)
    vp, i = ctypes.c_void_p, ctypes.c_int
    for f in ("hevc_transform_quant_4x4", "hevc_transform_quant_4x4_10"):
        getattr(L, f).argtypes = [vp, i, i, i, vp]
    for f in ("hevc_dequant_itransform_4x4", "hevc_dequant_itransform_4x4_10"):
        getattr(L, f).argtypes = [vp, i, i, vp]
    L.hevc_transform_quant_8x8.argtypes = [vp, i, i, i, vp]
    L.hevc_dequant_itransform_8x8.argtypes = [vp, i, i, vp]
    L.refshim_hevc_build_hpel.argtypes = [vp, i, i, ctypes.POINTER(vp)]
    return L


def _residuals(rs, n, size, bit_depth):
    lim = (1 << bit_depth) - 1
    x = rs.integers(-lim, lim + 1, (n, size)).astype(np.int16)
    x[: n // 16] = 0                                               # zero blocks
    x[n // 16: n // 8] = rs.integers(-lim, lim + 1, (n // 8 - n // 16, 1))  # flat blocks
    x[n // 8: n // 8 + 8] = rs.choice([-32768, 32767, -32767], (8, size))  # saturating extremes
    return np.ascontiguousarray(x)


def _levels(rs, n, size):
    c = (rs.integers(-40, 41, (n, size)) * (rs.random((n, size)) < 0.3)).astype(np.int16)
    c[: n // 16] = 0
    c[n // 16: n // 16 + 8] = rs.choice([-32768, 32767, 1000, -1000], (8, size))
    return np.ascontiguousarray(c)


def _gpu_run(fn, src, out_cols, *args):
    import torch
    s = torch.from_numpy(src).cuda()
    o = torch.full((src.shape[0], out_cols), -7, dtype=torch.int16, device="cuda")
    fn(s, o, *args)
    torch.cuda.synchronize()
    return o.cpu().numpy()


@needs_ref
@pytest.mark.parametrize("bit_depth,qps", [(8, [0, 7, 22, 27, 37, 51, 60, -3]), (10, [0, 12, 30, 45, 57, 63, 70])])
@pytest.mark.parametrize("use_dst", [0, 1])
@pytest.mark.parametrize("round_q12", [0, 2, 4, 6, 12])
def test_transform_quant_4x4(gpu, bit_depth, qps, use_dst, round_q12):
    L = _ref()
    f = L.hevc_transform_quant_4x4 if bit_depth == 8 else L.hevc_transform_quant_4x4_10
    rs = np.random.Generator(np.random.PCG64(bit_depth * 100 + use_dst * 10 + round_q12))
    x = _residuals(rs, 1024, 16, bit_depth)
    for qp in qps:
        got = _gpu_run(gpu.hevc_transform_quant_4x4, x, 16, qp, use_dst, round_q12, bit_depth)
        want = np.zeros_like(x)
        for b in range(x.shape[0]):
            f(x[b].ctypes.data, qp, use_dst, round_q12, want[b].ctypes.data)
        np.testing.assert_array_equal(got, want, err_msg=f"qp {qp}")


@needs_ref
@pytest.mark.parametrize("bit_depth,qps", [(8, [0, 5, 22, 27, 37, 51]), (10, [0, 12, 30, 45, 63, 70])])
@pytest.mark.parametrize("use_dst", [0, 1])
def test_dequant_itransform_4x4(gpu, bit_depth, qps, use_dst):
    L = _ref()
    f = L.hevc_dequant_itransform_4x4 if bit_depth == 8 else L.hevc_dequant_itransform_4x4_10
    rs = np.random.Generator(np.random.PCG64(bit_depth * 7 + use_dst))
    c = _levels(rs, 1024, 16)
    for qp in qps:
        got = _gpu_run(gpu.hevc_dequant_itransform_4x4, c, 16, qp, use_dst, bit_depth)
        want = np.zeros_like(c)
        for b in range(c.shape[0]):
            f(c[b].ctypes.data, qp, use_dst, want[b].ctypes.data)
        np.testing.assert_array_equal(got, want, err_msg=f"qp {qp}")


@needs_ref
@pytest.mark.parametrize("bit_depth,qps", [(8, [0, 9, 22, 27, 37, 51, 63, 70]), (10, [0, 12, 34, 49, 63])])
@pytest.mark.parametrize("round_q12", [0, 4, 6])
def test_transform_quant_8x8(gpu, bit_depth, qps, round_q12):
    L = _ref()
    rs = np.random.Generator(np.random.PCG64(bit_depth * 31 + round_q12))
    x = _residuals(rs, 512, 64, bit_depth)
    for qp in qps:
        got = _gpu_run(gpu.hevc_transform_quant_8x8, x, 64, qp, round_q12, bit_depth)
        want = np.zeros_like(x)
        for b in range(x.shape[0]):
            L.hevc_transform_quant_8x8(x[b].ctypes.data, qp, bit_depth, round_q12, want[b].ctypes.data)
        np.testing.assert_array_equal(got, want, err_msg=f"qp {qp}")


@needs_ref
@pytest.mark.parametrize("bit_depth,qps", [(8, [0, 9, 22, 27, 37, 51, 63]), (10, [0, 12, 34, 49, 63, 70])])
def test_dequant_itransform_8x8(gpu, bit_depth, qps):
    L = _ref()
    rs = np.random.Generator(np.random.PCG64(bit_depth * 3))
    c = _levels(rs, 512, 64)
    for qp in qps:
        got = _gpu_run(gpu.hevc_dequant_itransform_8x8, c, 64, qp, bit_depth)
        want = np.zeros_like(c)
        for b in range(c.shape[0]):
            L.hevc_dequant_itransform_8x8(c[b].ctypes.data, qp, bit_depth, want[b].ctypes.data)
        np.testing.assert_array_equal(got, want, err_msg=f"qp {qp}")


@needs_ref
@pytest.mark.parametrize("w,h", [(16, 16), (64, 48), (200, 120), (1920, 1088)])
def test_build_hpel(gpu, w, h):
    import torch
    L = _ref()
    rs = np.random.Generator(np.random.PCG64(w + h))
    recon = np.clip(128 + 60 * rs.standard_normal((h, w)), 0, 255).astype(np.uint8)
    recon[: h // 4] = rs.integers(0, 256, (h // 4, w))  # hard edges for the filters
    M = 16
    rows, cols = h + 2 * M, w + 2 * M
    want = [np.zeros((rows, cols), np.uint8) for _ in range(4)]
    ptrs = (ctypes.c_void_p * 4)(*[p.ctypes.data for p in want])
    assert L.refshim_hevc_build_hpel(recon.ctypes.data, w, h, ptrs) == M
    pitch = (w + 127) // 128 * 128
    dev = torch.zeros((h, pitch), dtype=torch.uint8, device="cuda")
    dev[:, :w] = torch.from_numpy(recon)
    ppitch = (cols + 127) // 128 * 128
    planes = torch.full((4, rows, ppitch), 7, dtype=torch.uint8, device="cuda")
    gpu.hevc_build_hpel(dev, w, h, M, planes)
    torch.cuda.synchronize()
    got = planes.cpu().numpy()
    for k, name in enumerate(("I", "H", "V", "HV")):
        np.testing.assert_array_equal(got[k, :, :cols], want[k], err_msg=f"plane {name}")
    assert (got[:, :, cols:] == 7).all(), "wrote past the plane width"


def test_rejects_bad_arguments(gpu):
    import torch
    x = torch.zeros((4, 16), dtype=torch.int16, device="cuda")
    L = gpu.lib()
    assert L.b200enc_hevc_transform_quant_4x4(gpu._p(x), gpu._p(x), 4, 27, 0, 4, 9, None) == -1  # bit depth
    assert L.b200enc_hevc_transform_quant_4x4(gpu._p(x), gpu._p(x), 4, 27, 0, 13, 8, None) == -1  # rounding
    assert L.b200enc_hevc_dequant_itransform_4x4(gpu._p(x), gpu._p(x), 4, 52, 0, 8, None) == -1  # 8-bit QP
    assert L.b200enc_hevc_transform_quant_4x4(gpu._p(x), gpu._p(x), 0, 27, 0, 4, 8, None) == 0   # empty batch


@needs_ref
@pytest.mark.parametrize("w,h,qpel,seed", [(320, 192, 1, 1), (320, 192, 0, 2), (200, 120, 1, 3), (64, 64, 1, 4)])
def test_motion_search(gpu, w, h, qpel, seed):
    """Every 8x8 CU of a frame, with predictors and starting points spread
    from the true motion to far outside the picture."""
    import torch
    from b200enc import synth
    L = _ref()
    L.refshim_hevc_motion_search.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    seq = synth.Sequence(w, h, seed=seed, pan=True)
    ref = np.ascontiguousarray(seq.frame(0)[0])
    src = np.ascontiguousarray(seq.frame(1)[0])
    M = 16
    rows, cols = h + 2 * M, w + 2 * M
    planes_h = [np.zeros((rows, cols), np.uint8) for _ in range(4)]
    ptrs = (ctypes.c_void_p * 4)(*[p.ctypes.data for p in planes_h])
    L.refshim_hevc_build_hpel(ref.ctypes.data, w, h, ptrs)
    rs = np.random.Generator(np.random.PCG64(seed))
    cus = [(x, y) for y in range(0, h - 7, 8) for x in range(0, w - 7, 8)]
    jobs = np.zeros(len(cus) + 2, gpu.HEVC_ME_JOB)
    for j, (x, y) in enumerate(cus):
        jobs[j]["cu_x"], jobs[j]["cu_y"] = x, y
        jobs[j]["mvp"] = rs.integers(-40, 41, (2, 2))
        ns = int(rs.integers(0, 17))
        st = rs.integers(-40, 41, (16, 2))
        st[::5] = rs.integers(-600, 601, (4, 2))[: len(st[::5])]  # far away: clamped to the margin
        jobs[j]["starts"] = st
        jobs[j]["n_starts"] = ns
        jobs[j]["lambda_q8"] = int(rs.integers(0, 4000))
    jobs[-2]["cu_x"], jobs[-2]["cu_y"] = w - 4, 0     # outside: rejected in the kernel
    jobs[-1]["cu_x"], jobs[-1]["cu_y"] = 0, h
    src_d = torch.from_numpy(src).cuda()
    ppitch = (cols + 127) // 128 * 128
    planes = torch.zeros((4, rows, ppitch), dtype=torch.uint8, device="cuda")
    for k in range(4):
        planes[k, :, :cols] = torch.from_numpy(planes_h[k])
    jobs_d = torch.from_numpy(jobs.view(np.uint8)).cuda()
    res_d = torch.zeros(len(jobs) * gpu.HEVC_ME_RESULT.itemsize, dtype=torch.uint8, device="cuda")
    gpu.hevc_motion_search(src_d, w, h, planes, M, qpel, jobs_d, res_d)
    torch.cuda.synchronize()
    got = res_d.cpu().numpy().view(gpu.HEVC_ME_RESULT)
    for j, (x, y) in enumerate(cus):
        mv = np.zeros(2, np.int16)
        idx, cost, sad = ctypes.c_int(), ctypes.c_int64(), ctypes.c_uint32()
        mvp = np.ascontiguousarray(jobs[j]["mvp"].reshape(-1))
        st = np.ascontiguousarray(jobs[j]["starts"].reshape(-1))
        L.refshim_hevc_motion_search(ptrs, src.ctypes.data, w, h, qpel, x, y, mvp.ctypes.data, st.ctypes.data,
                                     int(jobs[j]["n_starts"]), int(jobs[j]["lambda_q8"]), mv.ctypes.data,
                                     ctypes.byref(idx), ctypes.byref(cost), ctypes.byref(sad))
        g = got[j]
        assert (tuple(g["mv"]), int(g["mvp_idx"]), int(g["cost_q8"]), int(g["sad"])) == \
            (tuple(mv), idx.value, cost.value, sad.value), f"CU ({x},{y})"
    assert (got[-2]["sad"], got[-1]["sad"]) == (0xFFFFFFFF, 0xFFFFFFFF)


@needs_ref
@pytest.mark.parametrize("w,h,slices", [(64, 48, [0]), (200, 120, [0, 48]), (1920, 1088, [0, 272, 544, 816])])
def test_choose_luma_mode(gpu, w, h, slices):
    """Every 4x4 PU of a picture against a fixed reconstruction, including
    picture edges, CTU/CU/PU z-order availability and slice starts."""
    import torch
    L = _ref()
    L.hevc_choose_luma_mode.restype = ctypes.c_int
    L.hevc_choose_luma_mode.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    rs = np.random.Generator(np.random.PCG64(w * h))
    src = np.clip(128 + 50 * rs.standard_normal((h, w)), 0, 255).astype(np.uint8)
    rec = np.clip(src.astype(int) + rs.integers(-6, 7, (h, w)), 0, 255).astype(np.uint8)
    rec[h // 3: h // 3 + 8] = 255  # strong edges exercise the clipped H/V edge filters
    pus = [(x, y) for y in range(0, h, 4) for x in range(0, w, 4)]
    if w > 256:
        pus = pus[:: 7]
    jobs = np.array([(x, y, max(sy for sy in slices if sy <= y)) for x, y in pus] + [(w - 2, 0, 0), (0, h, 0)],
                    np.int32)
    modes = torch.full((len(jobs),), -5, dtype=torch.int32, device="cuda")
    preds = torch.zeros((len(jobs), 16), dtype=torch.uint8, device="cuda")
    gpu.hevc_choose_luma_mode(torch.from_numpy(src).cuda(), torch.from_numpy(rec).cuda(), w, h,
                              torch.from_numpy(jobs).cuda(), modes, preds)
    torch.cuda.synchronize()
    gm, gp = modes.cpu().numpy(), preds.cpu().numpy()
    for j, (x, y, ym) in enumerate(jobs[:-2]):
        pred = np.zeros(16, np.uint8)
        m = L.hevc_choose_luma_mode(int(ym), src.ctypes.data, rec.ctypes.data, w, w, h, int(x), int(y),
                                    pred.ctypes.data)
        assert gm[j] == m, f"PU ({x},{y}) mode"
        np.testing.assert_array_equal(gp[j], pred, err_msg=f"PU ({x},{y}) prediction")
    assert gm[-2] == -1 and gm[-1] == -1
