"""ctypes front end of the CPU oracle (oracle.c) and of the reference's own C
compiled into oracle/_ref (ref_shim.c + the reference sources).

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline legs may import this module; the product library never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libh264ref.so")
REF_DEC = os.path.join(HERE, "_ref", "h264dec")

_u8p = ctypes.POINTER(ctypes.c_uint8)


class Frame(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int), ("H", ctypes.c_int), ("RW", ctypes.c_int), ("RH", ctypes.c_int),
                ("mbw", ctypes.c_int), ("mbh", ctypes.c_int), ("qp", ctypes.c_int), ("num_slices", ctypes.c_int),
                ("flags", ctypes.c_int)]


INTRA_CORNER_CHECK = 1


class MeParams(ctypes.Structure):
    _fields_ = [("range", ctypes.c_int), ("lambda_", ctypes.c_int), ("zero_thresh", ctypes.c_int)]


class Out(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_void_p), ("dc", ctypes.c_void_p), ("nz", ctypes.c_void_p),
                ("pred_mode", ctypes.c_void_p), ("mv", ctypes.c_void_p)]


def build():
    """Compiles liboracle.so and, where the reference sources exist, _ref/."""
    subprocess.run([os.path.join(HERE, "build.sh")], check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _lib = ctypes.CDLL(ORACLE_SO)
    return _lib


def ref_available():
    return os.path.exists(REF_SO)


CAVLC_SO = os.path.join(HERE, "_ref", "libcavlcref.so")
_cavlc = None


def cavlc_ref_available():
    return os.path.exists(CAVLC_SO)


def ref_cavlc_slice_data(mbw, mbh, qp, is_idr, start_mb, end_mb, levels, dc, nz, pred_modes, mvs,
                         quality_level=4, cap=None):
    """The reference's CAVLC slice data (encoder_h264.c's macroblock loop and
    encoders, cavlc.c) for macroblocks [start_mb, end_mb), from bit 0, with
    rbsp_trailing_bits: bytes."""
    global _cavlc
    if _cavlc is None:
        _cavlc = ctypes.CDLL(CAVLC_SO)
    cap = cap or (end_mb - start_mb) * 2560 + 4096
    out = np.zeros(cap, np.uint8)
    a = [np.ascontiguousarray(levels, np.int16), np.ascontiguousarray(dc, np.int32),
         np.ascontiguousarray(nz, np.uint32), np.ascontiguousarray(pred_modes, np.uint32),
         np.ascontiguousarray(mvs, np.int32)]
    n = _cavlc.refshim_cavlc_slice_data(mbw, mbh, qp, int(is_idr), quality_level, start_mb, end_mb,
                                        *[_p(x) for x in a], _p(out), cap)
    if n < 0:
        raise ValueError("slice data overflow")
    return out[:n].tobytes()


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
        _ref.refshim_sad16.restype = ctypes.c_uint32
    return _ref


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def frame(W, H, qp, num_slices=1, coded_clamp=True, corner_check=True):
    mbw, mbh = (W + 15) // 16, (H + 15) // 16
    RW, RH = (mbw * 16, mbh * 16) if coded_clamp else (W, H)
    return Frame(W, H, RW, RH, mbw, mbh, qp, num_slices, INTRA_CORNER_CHECK if corner_check else 0)


def alloc_outputs(mbs):
    return {
        "levels": np.zeros((mbs, 24, 16), np.int16),
        "dc": np.zeros((mbs, 24), np.int32),
        "nz": np.zeros((mbs, 24), np.uint32),
        "pred_mode": np.zeros((mbs,), np.uint32),
        "mv": np.zeros((mbs, 4), np.int32),
    }


def _out_struct(o):
    return Out(_p(o["levels"]), _p(o["dc"]), _p(o["nz"]), _p(o["pred_mode"]), _p(o["mv"]))


def me_frame(f, cur_y, ref_y, rng, lam, zero_thresh=512):
    """Plain full-search ME; cur_y/ref_y are 2-D uint8 arrays (pitch = shape[1])."""
    mv = np.zeros((f.mbw * f.mbh, 4), np.int32)
    lib().orc_me_frame(ctypes.byref(f), ctypes.byref(MeParams(rng, lam, zero_thresh)),
                       _p(cur_y), cur_y.shape[1], _p(ref_y), ref_y.shape[1], _p(mv))
    return mv


def me_refine(f, cur_y, ref_y, mbx, mby, imx, imy, int_sad):
    """Half/quarter-pel refine of the plain search around integer winner (imx, imy)."""
    o = np.zeros(4, np.int32)
    lib().orc_me_refine(ctypes.byref(f), _p(cur_y), cur_y.shape[1], _p(ref_y), ref_y.shape[1], int(mbx), int(mby),
                        int(imx), int(imy), ctypes.c_uint32(int(int_sad)), _p(o))
    return o


def me_rect_key(f, cur_y, ref_y, rng, lam, mbx, mby, x0, y0, x1, y1):
    """The plain search's key minimised over the integer MVs of [x0,x1] x [y0,y1]."""
    lib().orc_me_rect_key.restype = ctypes.c_uint32
    return int(lib().orc_me_rect_key(ctypes.byref(f), ctypes.byref(MeParams(rng, lam, -1)), _p(cur_y),
                                     cur_y.shape[1], _p(ref_y), ref_y.shape[1], int(mbx), int(mby), int(x0), int(y0),
                                     int(x1), int(y1)))


def p_frame(f, cur_y, cur_uv, ref_y, ref_uv, mv, rec_y, rec_uv):
    o = alloc_outputs(f.mbw * f.mbh)
    o["mv"][:] = mv
    lib().orc_p_frame(ctypes.byref(f), _p(cur_y), _p(cur_uv), cur_y.shape[1], _p(ref_y), _p(ref_uv), ref_y.shape[1],
                      _p(o["mv"]), ctypes.byref(_out_struct(o)), _p(rec_y), _p(rec_uv), rec_y.shape[1])
    return o


def p_frame_t8(f, cur_y, cur_uv, ref_y, ref_uv, mv, rec_y, rec_uv, t8):
    """The P chain with the 8x8 luma transform (t8 1: every macroblock, 2:
    chosen per macroblock); returns the outputs and the per-macroblock flags."""
    o = alloc_outputs(f.mbw * f.mbh)
    o["mv"][:] = mv
    flags = np.zeros(f.mbw * f.mbh, np.uint8)
    lib().orc_p_frame_t8(ctypes.byref(f), _p(cur_y), _p(cur_uv), cur_y.shape[1], _p(ref_y), _p(ref_uv),
                         ref_y.shape[1], _p(o["mv"]), ctypes.byref(_out_struct(o)), _p(rec_y), _p(rec_uv),
                         rec_y.shape[1], int(t8), _p(flags))
    return o, flags


def t8_choose(res):
    """1 when a macroblock's luma residual (int [16][16]) costs less under
    the 8x8 transform."""
    r = np.ascontiguousarray(res, np.int32).reshape(256)
    return int(lib().orc_t8_choose(_p(r)))


def i_frame(f, cur_y, cur_uv, rec_y, rec_uv):
    o = alloc_outputs(f.mbw * f.mbh)
    lib().orc_i_frame(ctypes.byref(f), _p(cur_y), _p(cur_uv), cur_y.shape[1], ctypes.byref(_out_struct(o)),
                      _p(rec_y), _p(rec_uv), rec_y.shape[1])
    return o


def i_frame_steps(f, cur_y, cur_uv, rec_y, rec_uv, order):
    """The I frame's macroblocks in the given order of raster indices (oracle.h)."""
    o = alloc_outputs(f.mbw * f.mbh)
    st = np.ascontiguousarray(order, np.int32)
    rc = lib().orc_i_frame_steps(ctypes.byref(f), _p(cur_y), _p(cur_uv), cur_y.shape[1], ctypes.byref(_out_struct(o)),
                                 _p(rec_y), _p(rec_uv), rec_y.shape[1], _p(st), len(st))
    if rc != 0:
        raise ValueError("macroblock outside the picture")
    return o


def set_threads(n):
    """Threads of the oracle's parallel loops (full search, P chain)."""
    lib().orc_set_threads(int(n))


def deblock(mbw, mbh, qp, is_intra, nz, mv, rec_y, rec_uv):
    lib().orc_deblock_frame(mbw, mbh, qp, int(is_intra), _p(np.ascontiguousarray(nz, np.uint32)),
                            _p(np.ascontiguousarray(mv, np.int32)), _p(rec_y), _p(rec_uv), rec_y.shape[1])


def deblock_t8(mbw, mbh, qp, is_intra, nz, t8, mv, rec_y, rec_uv):
    """Deblocking with the 8x8 transform in the macroblocks whose t8 byte is set."""
    lib().orc_deblock_frame_t8(mbw, mbh, qp, int(is_intra), _p(np.ascontiguousarray(nz, np.uint32)),
                               _p(np.ascontiguousarray(t8, np.uint8)), _p(np.ascontiguousarray(mv, np.int32)),
                               _p(rec_y), _p(rec_uv), rec_y.shape[1])


def deblock_steps(mbw, mbh, qp, is_intra, nz, mv, rec_y, rec_uv, steps):
    """The deblocking steps (2 * mb + dir) in the given order (oracle.h)."""
    st = np.ascontiguousarray(steps, np.int32)
    rc = lib().orc_deblock_steps(mbw, mbh, qp, int(is_intra), _p(np.ascontiguousarray(nz, np.uint32)),
                                 _p(np.ascontiguousarray(mv, np.int32)), _p(rec_y), _p(rec_uv), rec_y.shape[1],
                                 _p(st), len(st))
    if rc != 0:
        raise ValueError("deblocking step outside the picture")


def encode_frame(f, rng, lam, zero_thresh, is_intra, do_deblock, cur_y, cur_uv, ref_y, ref_uv, rec_y, rec_uv):
    o = alloc_outputs(f.mbw * f.mbh)
    lib().orc_encode_frame(ctypes.byref(f), ctypes.byref(MeParams(rng, lam, zero_thresh)), int(is_intra),
                           int(do_deblock), _p(cur_y), _p(cur_uv), cur_y.shape[1], _p(ref_y), _p(ref_uv),
                           ref_y.shape[1], ctypes.byref(_out_struct(o)), _p(rec_y), _p(rec_uv), rec_y.shape[1])
    return o


def intra16_luma_dc(dc_in, qp):
    lib().orc_intra16_luma_dc_transform.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    a = np.ascontiguousarray(dc_in, np.int32)
    out = np.zeros(16, np.int32)
    pre = np.zeros(16, np.int32)
    lib().orc_intra16_luma_dc_transform(_p(a), qp, _p(out), _p(pre))
    return out, pre


def interp_luma(ref_y, RW, RH, qx, qy):
    return lib().orc_interp_luma_qpel(_p(ref_y), ref_y.shape[1], int(RW), int(RH), int(qx), int(qy))


# ---------------------------------------------------------------- reference

def fwd_quant8(res, qp, intra):
    """Forward 8x8 transform + quantisation of int16 [n][64] residual blocks."""
    res = np.ascontiguousarray(res, np.int16).reshape(-1, 64)
    lev = np.zeros_like(res)
    for i in range(res.shape[0]):
        lib().orc_fwd_quant8(_p(res[i]), _p(lev[i]), qp, int(intra))
    return lev


def dequant_idct8_add(lev, pred, qp):
    """Scaling + inverse 8x8 + add onto uint8 [8][8] predictions ([n][8][8])."""
    lev = np.ascontiguousarray(lev, np.int16).reshape(-1, 64)
    out = np.ascontiguousarray(pred, np.uint8).reshape(-1, 8, 8).copy()
    for i in range(lev.shape[0]):
        lib().orc_dequant_idct8_add(_p(lev[i]), _p(out[i]), 8, qp)
    return out


def ref_idct8_add(lev, pred, qp):
    """The reference decoder's h264d_idct8_add on the same blocks."""
    lev = np.ascontiguousarray(lev, np.int16).reshape(-1, 64).copy()
    out = np.ascontiguousarray(pred, np.uint8).reshape(-1, 8, 8).copy()
    for i in range(lev.shape[0]):
        ref().refshim_idct8_add(_p(out[i]), 8, _p(lev[i]), qp)
    return out


def ref_deblock_t8(mbw, mbh, qp, is_intra, nz, t8, mv, rec_y, rec_uv):
    """The reference decoder's deblocking with 8x8-transform macroblocks (t8)."""
    r = ref().refshim_deblock_nv12_t8(mbw, mbh, qp, int(is_intra), _p(np.ascontiguousarray(nz, np.uint32)),
                                      _p(np.ascontiguousarray(t8, np.uint8)), _p(np.ascontiguousarray(mv, np.int32)),
                                      _p(rec_y), _p(rec_uv), rec_y.shape[1])
    if r != 0:
        raise RuntimeError("refshim_deblock_nv12_t8 failed")


def ref_deblock(mbw, mbh, qp, is_intra, nz, mv, rec_y, rec_uv):
    r = ref().refshim_deblock_nv12(mbw, mbh, qp, int(is_intra), _p(np.ascontiguousarray(nz, np.uint32)),
                                   _p(np.ascontiguousarray(mv, np.int32)), _p(rec_y), _p(rec_uv), rec_y.shape[1])
    assert r == 0


def ref_mc_luma(plane, pw, ph, qx, qy, w=16, h=16):
    dst = np.zeros((h, w), np.uint8)
    ref().refshim_mc_luma(_p(plane), plane.shape[1], pw, ph, qx, qy, w, h, _p(dst), w)
    return dst


def ref_mc_chroma(uv, cw, chh, plane, ex, ey, w=8, h=8):
    dst = np.zeros((h, w), np.uint8)
    ref().refshim_mc_chroma_nv12(_p(uv), uv.shape[1], cw, chh, plane, ex, ey, w, h, _p(dst), w)
    return dst


def ref_idct4_add(dst, block, qp, dc_ready):
    b = np.ascontiguousarray(block, np.int16).copy()
    ref().refshim_idct4_add(_p(dst), dst.shape[1], _p(b), qp, int(dc_ready))


def ref_sad16(a, b):
    return ref().refshim_sad16(_p(a), a.shape[1], _p(b), b.shape[1])


def ref_intra16_luma_dc(dc_in, qp):
    a = np.ascontiguousarray(dc_in, np.int32)
    out = np.zeros(16, np.int32)
    pre = np.zeros(16, np.int32)
    ref().refshim_intra16_luma_dc(_p(a), qp, _p(out), _p(pre))
    return out, pre


def ref_cpu_me(cur_y, ref_y, W, H, radius, threads=1):
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    mv = np.zeros((mbs, 4), np.int32)
    r = ref().refshim_cpu_me(_p(cur_y), cur_y.shape[1], _p(ref_y), ref_y.shape[1], W, H, radius, threads, _p(mv))
    assert r == 0
    return mv


def ref_full_search_int(cur_y, W, H, ref_y, RW, RH, rng, lam, row0=0, row1=None, threads=0):
    """The plain full search's integer stage at the reference's AVX2 SAD speed."""
    mbw, mbh = (W + 15) // 16, (H + 15) // 16
    row1 = mbh if row1 is None else row1
    dx = np.zeros(mbw * mbh, np.int32)
    dy = np.zeros(mbw * mbh, np.int32)
    sad = np.zeros(mbw * mbh, np.uint32)
    r = ref().refshim_full_search_int(_p(cur_y), cur_y.shape[1], W, H, _p(ref_y), ref_y.shape[1], RW, RH, mbw,
                                      row0, row1, rng, lam, threads, _p(dx), _p(dy), _p(sad))
    assert r == 0
    return dx, dy, sad
