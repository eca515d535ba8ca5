"""Main10 (10-bit) instances of the HEVC motion-search and intra primitives
(b200enc_hevc_build_hpel_10, _motion_search_10, _choose_luma_mode_10)
against the reference's own BIT_DEPTH 10 template instances, compiled from
its sources (oracle/_ref/libhevcref.so: build_hpel_10 and motion_search_10
of encoder_h265.c through oracle/hevc_shim.c, hevc_choose_luma_mode_10 of
hevc_intra.c as is), bit for bit, on P010-range content (samples 64..940 with
film-grain noise, as the 2160p Main10 workload describes) at 416x240 and
3840x2160.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEVC_SO = os.path.join(ROOT, "oracle", "_ref", "libhevcref.so")
needs_ref = pytest.mark.skipif(not os.path.exists(HEVC_SO), reason="reference HEVC routines not built")
SIZES = [(416, 240), (3840, 2160)]


def _ref():
    L = ctypes.CDLL(HEVC_SO)
    vp, i = ctypes.c_void_p, ctypes.c_int
    L.refshim_hevc_build_hpel_10.argtypes = [vp, i, i, ctypes.POINTER(vp)]
    L.refshim_hevc_motion_search_10.argtypes = [ctypes.POINTER(vp), vp, i, i, i, i, i, vp, vp, i, i, vp, vp, vp, vp]
    L.hevc_choose_luma_mode_10.restype = i
    L.hevc_choose_luma_mode_10.argtypes = [i, vp, vp, i, i, i, i, i, vp]
    return L


def _p010_frames(w, h, seed, n=2):
    """n frames of 10-bit samples in 64..940: the seeded 8-bit generator's
    content (panning, moving rectangles) mapped to the 10-bit range plus
    film-grain noise of sigma 12."""
    from b200enc import synth
    seq = synth.Sequence(w, h, seed=seed, pan=True)
    rs = np.random.Generator(np.random.PCG64(seed))
    out = []
    for t in range(n):
        y8 = seq.frame(t)[0].astype(np.float64)
        v = 64 + y8 * (876.0 / 255.0) + rs.normal(0.0, 12.0, size=y8.shape)
        out.append(np.clip(np.rint(v), 64, 940).astype(np.uint16))
    return out


def _ref_planes(L, rec, w, h):
    M = 16
    rows, cols = h + 2 * M, w + 2 * M
    planes = [np.zeros((rows, cols), np.uint16) for _ in range(4)]
    ptrs = (ctypes.c_void_p * 4)(*[p.ctypes.data for p in planes])
    assert L.refshim_hevc_build_hpel_10(rec.ctypes.data, w, h, ptrs) == M
    return planes, ptrs


def _dev16(a, pitch=None):
    import torch
    h, w = a.shape
    pitch = pitch or (w + 63) // 64 * 64
    d = torch.zeros((h, pitch), dtype=torch.int16, device="cuda")
    d[:, :w] = torch.from_numpy(a.view(np.int16))
    return d


@needs_ref
@pytest.mark.parametrize("w,h", SIZES)
def test_build_hpel_10(gpu, w, h):
    import torch
    L = _ref()
    rec = _p010_frames(w, h, seed=w + 1, n=1)[0]
    rec[: h // 5, : w // 3] = np.where(np.arange(w // 3) % 7 < 3, 940, 64)  # hard edges: the clip at 1023
    want, _ = _ref_planes(L, rec, w, h)
    M = 16
    rows, cols = h + 2 * M, w + 2 * M
    ppitch = (cols + 63) // 64 * 64
    planes = torch.full((4, rows, ppitch), 7, dtype=torch.int16, device="cuda")
    gpu.hevc_build_hpel(_dev16(rec), w, h, M, planes)
    torch.cuda.synchronize()
    got = planes.cpu().numpy().view(np.uint16)
    for k, name in enumerate(("I", "H", "V", "HV")):
        np.testing.assert_array_equal(got[k, :, :cols], want[k], err_msg=f"plane {name}")
    assert (got[:, :, cols:] == 7).all(), "wrote past the plane width"
    assert got[1:].max() <= 1023


@needs_ref
@pytest.mark.parametrize("w,h,qpel", [(416, 240, 1), (416, 240, 0), (3840, 2160, 1)])
def test_motion_search_10(gpu, w, h, qpel):
    """8x8 CUs of a 10-bit frame (every CU at 416x240, every 11th at 2160p),
    predictors and starting points from the true motion to far outside."""
    import torch
    L = _ref()
    ref, src = _p010_frames(w, h, seed=w + h + qpel)
    planes_h, ptrs = _ref_planes(L, ref, w, h)
    M = 16
    rows, cols = h + 2 * M, w + 2 * M
    rs = np.random.Generator(np.random.PCG64(w * 3 + qpel))
    cus = [(x, y) for y in range(0, h - 7, 8) for x in range(0, w - 7, 8)]
    if w > 1000:
        cus = cus[::11]
    jobs = np.zeros(len(cus) + 1, gpu.HEVC_ME_JOB)
    for j, (x, y) in enumerate(cus):
        jobs[j]["cu_x"], jobs[j]["cu_y"] = x, y
        jobs[j]["mvp"] = rs.integers(-40, 41, (2, 2))
        st = rs.integers(-40, 41, (16, 2))
        st[::5] = rs.integers(-600, 601, (4, 2))[: len(st[::5])]
        jobs[j]["starts"] = st
        jobs[j]["n_starts"] = int(rs.integers(0, 17))
        jobs[j]["lambda_q8"] = int(rs.integers(0, 4000))
    jobs[-1]["cu_x"], jobs[-1]["cu_y"] = w - 4, 0  # not a CU of the picture
    ppitch = (cols + 63) // 64 * 64
    planes = torch.zeros((4, rows, ppitch), dtype=torch.int16, device="cuda")
    for k in range(4):
        planes[k, :, :cols] = torch.from_numpy(planes_h[k].view(np.int16))
    jobs_d = torch.from_numpy(jobs.view(np.uint8)).cuda()
    res_d = torch.zeros(len(jobs) * gpu.HEVC_ME_RESULT.itemsize, dtype=torch.uint8, device="cuda")
    gpu.hevc_motion_search(_dev16(src), w, h, planes, M, qpel, jobs_d, res_d)
    torch.cuda.synchronize()
    got = res_d.cpu().numpy().view(gpu.HEVC_ME_RESULT)
    for j, (x, y) in enumerate(cus):
        mv = np.zeros(2, np.int16)
        idx, cost, sad = ctypes.c_int(), ctypes.c_int64(), ctypes.c_uint32()
        mvp = np.ascontiguousarray(jobs[j]["mvp"].reshape(-1))
        st = np.ascontiguousarray(jobs[j]["starts"].reshape(-1))
        L.refshim_hevc_motion_search_10(ptrs, src.ctypes.data, w, h, qpel, x, y, mvp.ctypes.data, st.ctypes.data,
                                        int(jobs[j]["n_starts"]), int(jobs[j]["lambda_q8"]), mv.ctypes.data,
                                        ctypes.byref(idx), ctypes.byref(cost), ctypes.byref(sad))
        g = got[j]
        assert (tuple(g["mv"]), int(g["mvp_idx"]), int(g["cost_q8"]), int(g["sad"])) == \
            (tuple(mv), idx.value, cost.value, sad.value), f"CU ({x},{y})"
    assert got[-1]["sad"] == 0xFFFFFFFF


@needs_ref
@pytest.mark.parametrize("w,h,slices", [(416, 240, [0, 96]), (3840, 2160, [0, 544, 1088, 1632])])
def test_choose_luma_mode_10(gpu, w, h, slices):
    """4x4 PUs of a 10-bit picture (every PU at 416x240, every 13th at
    2160p), including the picture's first PU (no neighbour: fill 512), strong
    edges (the clipped H/V edge filters) and slice starts."""
    import torch
    L = _ref()
    src = _p010_frames(w, h, seed=w + 7, n=1)[0]
    rs = np.random.Generator(np.random.PCG64(w * h + 1))
    rec = np.clip(src.astype(int) + rs.integers(-20, 21, (h, w)), 0, 1023).astype(np.uint16)
    rec[h // 3: h // 3 + 8] = 1023
    rec[h // 2: h // 2 + 4] = 0
    pus = [(x, y) for y in range(0, h, 4) for x in range(0, w, 4)]
    if w > 1000:
        pus = pus[::13]
    jobs = np.array([(x, y, max(sy for sy in slices if sy <= y)) for x, y in pus] + [(w - 2, 0, 0)], np.int32)
    modes = torch.full((len(jobs),), -5, dtype=torch.int32, device="cuda")
    preds = torch.zeros((len(jobs), 16), dtype=torch.int16, device="cuda")
    gpu.hevc_choose_luma_mode(_dev16(src), _dev16(rec), w, h, torch.from_numpy(jobs).cuda(), modes, preds)
    torch.cuda.synchronize()
    gm, gp = modes.cpu().numpy(), preds.cpu().numpy().view(np.uint16)
    for j, (x, y, ym) in enumerate(jobs[:-1]):
        pred = np.zeros(16, np.uint16)
        m = L.hevc_choose_luma_mode_10(int(ym), src.ctypes.data, rec.ctypes.data, w, w, h, int(x), int(y),
                                       pred.ctypes.data)
        assert gm[j] == m, f"PU ({x},{y}) mode"
        np.testing.assert_array_equal(gp[j], pred, err_msg=f"PU ({x},{y}) prediction")
    assert gm[-1] == -1


def test_10bit_entry_points_reject_bad_arguments(gpu):
    import torch
    L = gpu.lib()
    x = torch.zeros((64, 64), dtype=torch.int16, device="cuda")
    p = gpu._p(x)
    assert L.b200enc_hevc_build_hpel_10(p, 8, 16, 16, 16, p, p, p, p, 48, None) == -1   # pitch < w
    assert L.b200enc_hevc_build_hpel_10(p, 16, 16, 16, 16, p, p, p, p, 40, None) == -1  # plane pitch < w + 2M
    assert L.b200enc_hevc_motion_search_10(p, 16, 16, 16, p, p, p, p, 48, 8, 1, p, 1, p, None) == -1  # margin < 10
    assert L.b200enc_hevc_choose_luma_mode_10(p, 16, p, 16, 3, 16, p, 1, p, p, None) == -1  # width < 4
    assert L.b200enc_hevc_motion_search_10(p, 16, 16, 16, p, p, p, p, 48, 16, 1, p, 0, p, None) == 0  # no jobs
