"""Pins the CPU oracle (oracle/oracle.c) against the reference's own C code.

Golden vectors in tests/golden/ were produced by the reference functions
(tests/golden/make_golden.py); where the reference library is built here the
tests also compare live on fresh seeded inputs. CPU only.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def test_intra16_dc_transpose_fixture(oracle_mod):
    # approach1-compute-encoder/tests/test_encode.c:60-96: the array handed
    # to CAVLC is the transpose of the quantized Hadamard output, and the
    # fixture is asymmetric.
    g = _load("dc_transpose.npz")
    out, pre = oracle_mod.intra16_luma_dc(g["dc_in"][0], int(g["qp"][0]))
    P = pre.reshape(4, 4)
    assert (P != P.T).any(), "fixture must give an asymmetric pre-transpose array"
    assert np.array_equal(out.reshape(4, 4), P.T)
    np.testing.assert_array_equal(out, g["dc_out"][0])
    np.testing.assert_array_equal(pre, g["pre"][0])


def test_intra16_dc_seeded(oracle_mod):
    g = _load("dc_transpose.npz")
    for a, q, o_ref, p_ref in zip(g["dc_in"], g["qp"], g["dc_out"], g["pre"]):
        out, pre = oracle_mod.intra16_luma_dc(a, int(q))
        np.testing.assert_array_equal(out, o_ref)
        np.testing.assert_array_equal(pre, p_ref)


def test_sad_kats(oracle_mod):
    # approach1-compute-encoder/tests/test_cpu_simd_me.c:16-43
    lib = oracle_mod.lib()
    a = np.full((16, 16), 128, np.uint8)
    b = np.full((16, 16), 128, np.uint8)
    sad = lambda x, y: lib.orc_sad16(oracle_mod._p(x), x.shape[1], oracle_mod._p(y), y.shape[1]) & 0xffffffff
    assert sad(a, b) == 0
    b[:] = 138
    assert sad(a, b) == 16 * 16 * 10
    ca = np.full((32, 32), 50, np.uint8)
    cb = np.full((32, 32), 60, np.uint8)
    assert sad(ca, cb) == 16 * 16 * 10
    g = _load("sad.npz")
    for x, y, s in zip(g["a"], g["b"], g["sad"]):
        assert sad(np.ascontiguousarray(x), np.ascontiguousarray(y)) == int(s)


def test_me_shift_kat(oracle_mod):
    # approach1-compute-encoder/tests/test_cpu_simd_me.c:45-106: a pattern
    # shifted by (2,2) in the reference is found at MV (8,8) quarter-pel;
    # a static MB keeps MV (0,0).
    W = H = 64
    ref = np.full((H, W), 100, np.uint8)
    cur = np.full((H, W), 100, np.uint8)
    yy, xx = np.mgrid[0:16, 0:16]
    cur[16:32, 16:32] = ((xx * 13 + yy * 7 + 40) % 256).astype(np.uint8)
    ref[18:34, 18:34] = cur[16:32, 16:32]
    f = oracle_mod.frame(W, H, 26)
    for rng in (16, 32):
        mv = oracle_mod.me_frame(f, cur, ref, rng, 5)
        assert tuple(mv[0, :2]) == (0, 0)
        assert tuple(mv[1 * 4 + 1, :2]) == (8, 8)
        assert mv[5, 2] == 0


def test_mc_every_phase(oracle_mod):
    g = _load("mc.npz")
    plane = np.ascontiguousarray(g["plane"])
    for (qx, qy), blk in zip(g["pos"], g["luma"]):
        got = np.array([[oracle_mod.interp_luma(plane, 48, 40, qx + 4 * x, qy + 4 * y) for x in range(16)]
                        for y in range(16)], np.uint8)
        np.testing.assert_array_equal(got, blk, err_msg=f"luma MC at ({qx},{qy})")
    uv = np.ascontiguousarray(g["uv"])
    lib = oracle_mod.lib()
    for (pl, ex, ey), blk in zip(g["cpos"], g["chroma"]):
        got = np.array([[lib.orc_interp_chroma(oracle_mod._p(uv), 48, 48, 40, int(pl), int(ex) + 8 * x, int(ey) + 8 * y)
                         for x in range(8)] for y in range(8)], np.uint8)
        np.testing.assert_array_equal(got, blk, err_msg=f"chroma MC plane {pl} at ({ex},{ey})")


def test_dequant_inverse(oracle_mod):
    g = _load("idct.npz")
    lib = oracle_mod.lib()
    import ctypes
    for lev, q, pred, rec in zip(g["levels"], g["qp"], g["pred"], g["rec"]):
        d = np.array([lib.orc_dequant_ac(int(lev[p]), p, int(q)) for p in range(16)], np.int32)
        r = np.zeros(16, np.int32)
        lib.orc_inverse_4x4(d.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p))
        got = np.clip(pred.astype(np.int32) + r.reshape(4, 4), 0, 255).astype(np.uint8)
        np.testing.assert_array_equal(got, rec, err_msg=f"qp {q}")


def test_deblock_against_reference_decoder(oracle_mod):
    g = _load("deblock.npz")
    changed = 0
    for i in range(int(g["n"])):
        c = {k: g[f"c{i}_{k}"] for k in ("mbw", "mbh", "qp", "intra", "y", "uv", "nz", "mv", "y_out", "uv_out")}
        y, uv = c["y"].copy(), c["uv"].copy()
        oracle_mod.deblock(int(c["mbw"]), int(c["mbh"]), int(c["qp"]), int(c["intra"]), c["nz"], c["mv"], y, uv)
        np.testing.assert_array_equal(y, c["y_out"], err_msg=f"luma case {i}")
        np.testing.assert_array_equal(uv, c["uv_out"], err_msg=f"chroma case {i}")
        changed += int((c["y_out"] != c["y"]).any())
    assert changed >= 4, "fixtures should exercise the filters"


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLD), "..", "oracle", "_ref", "libh264ref.so")),
                    reason="reference library not built here")
def test_full_search_integer_decision_vs_reference_sad(oracle_mod):
    """The oracle's exhaustive search and an independent loop over the
    reference's AVX2 cpu_simd_sad_16x16 pick the same integer vector."""
    from b200enc import synth
    seq = synth.Sequence(96, 64, seed=3)
    (y0, _), (y1, _) = seq.frame(0), seq.frame(1)
    f = oracle_mod.frame(96, 64, 26)
    for rng, lam in ((16, 5), (32, 8)):
        mv = oracle_mod.me_frame(f, y1, y0, rng, lam, zero_thresh=-1)
        dx, dy, sad = oracle_mod.ref_full_search_int(y1, 96, 64, y0, 96, 64, rng, lam)
        # the sub-pel refine moves at most 3/4 pel away from the integer pick
        assert np.all(np.abs(mv[:, 0] - 4 * dx) <= 3) and np.all(np.abs(mv[:, 1] - 4 * dy) <= 3)


def test_reference_live_deblock_and_mc(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference library not built here")
    rng = np.random.Generator(np.random.PCG64(7))
    for trial in range(6):
        mbw, mbh = int(rng.integers(1, 6)), int(rng.integers(1, 5))
        qp, intra = int(rng.integers(16, 52)), int(trial & 1)
        y = (np.clip(128 + 35 * rng.standard_normal((mbh * 16, mbw * 16)), 0, 255) // 6 * 6).astype(np.uint8)
        uv = np.clip(128 + 25 * rng.standard_normal((mbh * 8, mbw * 16)), 0, 255).astype(np.uint8)
        nz = rng.integers(0, 1 << 16, (mbw * mbh, 24)).astype(np.uint32) * (rng.random((mbw * mbh, 24)) < 0.3)
        mv = np.zeros((mbw * mbh, 4), np.int32)
        mv[:, :2] = rng.integers(-9, 10, (mbw * mbh, 2))
        a_y, a_uv, b_y, b_uv = y.copy(), uv.copy(), y.copy(), uv.copy()
        oracle_mod.deblock(mbw, mbh, qp, intra, nz.astype(np.uint32), mv, a_y, a_uv)
        oracle_mod.ref_deblock(mbw, mbh, qp, intra, nz.astype(np.uint32), mv, b_y, b_uv)
        np.testing.assert_array_equal(a_y, b_y)
        np.testing.assert_array_equal(a_uv, b_uv)
