"""Seeded inputs for the HEVC deblocking tests: one 4:2:0 picture with the
decoder-side maps b200enc_hevc_deblock takes (edge flags per 8x8 cell,
motion per 4x4, CBF per 4x4, QpY and lossless flags per min coding block,
slices and tiles per CTB), and a runner for the reference's filter
(oracle/_ref/libhevcfilt.so, the decoder's hevc_filter.c behind
oracle/hevc_filter_shim.c)."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FILT_SO = os.path.join(ROOT, "oracle", "_ref", "libhevcfilt.so")


def make_case(seed, width, height, bit_depth=8, log2_ctb=6, log2_min_cb=3, slices=1, tiles=1,
              lossless=0.0, intra=False, qp_range=(26, 51), cb_qp_offset=0, cr_qp_offset=0, pad=32,
              across_tiles=False, slice_params=None):
    """Returns a dict of host arrays and scalars describing one picture."""
    rs = np.random.Generator(np.random.PCG64(seed))
    maxv = (1 << bit_depth) - 1
    dt = np.uint8 if bit_depth == 8 else np.uint16

    def plane(h, w, block):
        # piecewise-constant blocks (steps at the block edges), smooth ramps
        # inside some blocks (strong-filter candidates), and noise patches
        # (decisions that fail)
        base = rs.integers(0, maxv + 1, ((h + block - 1) // block, (w + block - 1) // block))
        img = np.kron(base, np.ones((block, block)))[:h, :w].astype(np.int64)
        step = max(1, maxv // 64)
        img = (img // (8 * step)) * (8 * step)                    # fewer levels: small steps happen
        img += rs.integers(-step, step + 1, (h, w))                # mild texture
        ramp = rs.random((h // block + 1, w // block + 1)) < 0.3
        yy, xx = np.mgrid[0:h, 0:w]
        img += (np.kron(ramp, np.ones((block, block)))[:h, :w] * ((xx + yy) % block) * step).astype(np.int64)
        noisy = np.kron(rs.random((h // 32 + 1, w // 32 + 1)) < 0.1, np.ones((32, 32)))[:h, :w] > 0
        img[noisy] = rs.integers(0, maxv + 1, int(noisy.sum()))
        return np.clip(img, 0, maxv)

    W, H = width, height
    strides = [W + pad, W // 2 + pad, W // 2 + pad + 8]
    planes = []
    for c, (h, w) in enumerate(((H, W), (H // 2, W // 2), (H // 2, W // 2))):
        buf = rs.integers(0, maxv + 1, (h, strides[c])).astype(dt)   # padding: random, must survive
        buf[:, :w] = plane(h, w, 8 if c == 0 else 4).astype(dt)
        planes.append(np.ascontiguousarray(buf))

    ew = W // 8 + 1                                             # one spare cell a row (not read)
    eh = (H + 7) // 8
    e = np.zeros((eh, ew), np.uint8)
    e |= (rs.random((eh, ew)) < 0.75).astype(np.uint8) * 1
    e |= (rs.random((eh, ew)) < 0.75).astype(np.uint8) * 2
    e |= (rs.random((eh, ew)) < 0.5).astype(np.uint8) * 4
    e |= (rs.random((eh, ew)) < 0.5).astype(np.uint8) * 8
    e[:, W // 8:] = 0                                            # the spare cell: no edge there

    mpw, mph = W // 4 + 2, (H + 3) // 4
    mvf = None
    if not intra:
        mvf = np.zeros((mph, mpw), dtype=_mvf_dtype())
        flags = rs.choice([0, 1, 2, 3], (mph, mpw), p=[0.15, 0.4, 0.15, 0.3]).astype(np.uint8)
        # neighbours often alike (bS 0 happens), sometimes far apart
        mv = rs.integers(-6, 7, (mph, mpw, 2, 2)).astype(np.int16)
        same = rs.random((mph, mpw)) < 0.4
        mv[same] = 0
        mvf["mv"] = mv
        mvf["ref_poc"] = rs.choice([0, 1, 4], (mph, mpw, 2)).astype(np.int32)
        mvf["pred_flag"] = flags
    cbf = (rs.random((mph, mpw)) < 0.4).astype(np.uint8)

    mcw, mch = W >> log2_min_cb, H >> log2_min_cb
    qlo, qhi = qp_range
    qp = rs.integers(qlo, qhi + 1, (mch, mcw)).astype(np.int8)
    no_filter = (rs.random((mch, mcw)) < lossless).astype(np.uint8) if lossless > 0 else None

    cs = 1 << log2_ctb
    ctb_w, ctb_h = (W + cs - 1) // cs, (H + cs - 1) // cs
    n = ctb_w * ctb_h
    slice_of_ctb = None
    if slices > 1:
        cuts = np.sort(rs.choice(np.arange(1, n), slices - 1, replace=False))
        slice_of_ctb = np.zeros(n, np.int32)
        for k, c in enumerate(cuts):
            slice_of_ctb[c:] = k + 1
    sf = np.zeros(max(1, slices), dtype=_sf_dtype())
    if slice_params is None:
        sf["beta_offset"] = rs.integers(-6, 7, len(sf)) * 2
        sf["tc_offset"] = rs.integers(-6, 7, len(sf)) * 2
        sf["disabled"] = 0
        sf["across_slices"] = rs.integers(0, 2, len(sf))
        if len(sf) > 2:
            sf["disabled"][1] = 1
        sf[0]["beta_offset"], sf[0]["tc_offset"] = 0, 0
    else:
        for k, (b, t, d, a) in enumerate(slice_params):
            sf[k] = (b, t, d, a, (0, 0))
    tile_of_ctb = None
    if tiles > 1:
        tile_of_ctb = np.zeros((ctb_h, ctb_w), np.int32)
        cols = np.array_split(np.arange(ctb_w), tiles)
        for k, cset in enumerate(cols):
            tile_of_ctb[:, cset] = k
        tile_of_ctb = tile_of_ctb.reshape(-1)
    return dict(planes=planes, strides=strides, width=W, height=H, bit_depth=bit_depth, log2_ctb=log2_ctb,
                log2_min_cb=log2_min_cb, edges=e, edges_stride=ew, mvf=mvf, cbf=cbf, min_pu_width=mpw,
                qp_y=qp, no_filter=no_filter, slice_of_ctb=slice_of_ctb, slice_filter=sf, tile_of_ctb=tile_of_ctb,
                across_tiles=across_tiles, cb_qp_offset=cb_qp_offset, cr_qp_offset=cr_qp_offset)


def _mvf_dtype():
    return np.dtype([("mv", "<i2", (2, 2)), ("ref_poc", "<i4", (2,)), ("pred_flag", "u1"), ("pad", "u1", (3,))])


def _sf_dtype():
    return np.dtype([("beta_offset", "<i2"), ("tc_offset", "<i2"), ("disabled", "u1"), ("across_slices", "u1"),
                     ("pad", "u1", (2,))])


def params(b200enc, case, ptr, planes=None, slice_filter="default"):
    """The b200enc_hevc_deblock_t block for `case`, buffers turned into
    addresses by `ptr` (planes may be replaced, e.g. by copies)."""
    c = case
    pl = planes if planes is not None else c["planes"]
    sf = c["slice_filter"] if slice_filter == "default" else slice_filter
    return b200enc.hevc_deblock_params(
        ptr, pl, c["strides"], c["width"], c["height"], c["bit_depth"], c["bit_depth"], c["log2_ctb"],
        c["log2_min_cb"], c["edges"], c["edges_stride"], c["qp_y"], mvf=c["mvf"], cbf=c["cbf"],
        min_pu_width=c["min_pu_width"], no_filter=c["no_filter"], slice_of_ctb=c["slice_of_ctb"],
        slice_filter=sf, n_slice_filter=0 if sf is None else len(sf), tile_of_ctb=c["tile_of_ctb"],
        loop_filter_across_tiles=c["across_tiles"], cb_qp_offset=c["cb_qp_offset"], cr_qp_offset=c["cr_qp_offset"])


def np_ptr(a):
    return a.ctypes.data


def reference(b200enc, case, slice_filter="default"):
    """The reference filter over copies of the case's planes; returns them."""
    L = ctypes.CDLL(FILT_SO)
    L.refshim_hevc_deblock.argtypes = [ctypes.POINTER(b200enc.HevcDeblockParams)]
    out = [p.copy() for p in case["planes"]]
    q = params(b200enc, case, np_ptr, planes=out, slice_filter=slice_filter)
    assert L.refshim_hevc_deblock(ctypes.byref(q)) == 0
    return out
