"""Generates tests/golden/*.npz from the REFERENCE's own C functions.

Run in a container where the reference sources exist (oracle/Makefile builds
oracle/_ref/libh264ref.so from them). The outputs are committed, so the
tests can pin the oracle on machines without the reference. Each fixture
records the inputs (seeded) and the reference's outputs:
  dc_transpose.npz  encoder_h264.c h264_intra16_luma_dc_transform on the
                    tests/test_encode.c:60-96 fixture and on seeded inputs
  sad.npz           cpu_simd_me.c cpu_simd_sad_16x16 on the
                    test_cpu_simd_me.c:16-43 cases and seeded blocks
  mc.npz            h264_mc.c luma/chroma MC, every fractional phase
  idct.npz          h264_recon.c dequant + inverse 4x4 + add
  deblock.npz       h264_deblock.c on seeded pictures, intra and inter
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402


def main():
    oracle.build()
    assert oracle.ref_available(), "reference library not built (reference sources missing?)"
    rng = np.random.Generator(np.random.PCG64(0x243F6A88))

    # --- DC transpose / quant (A1/tests/test_encode.c:60-96 + seeded) ---
    fixture = np.array([16, 28, 40, 52, 64, 76, 88, 100, 112, 124, 136, 148, 160, 172, 184, 196], np.int32)
    ins, qps, outs, pres = [fixture], [26], [], []
    for _ in range(200):
        ins.append(rng.integers(-4080, 4081, 16).astype(np.int32))
        qps.append(int(rng.integers(0, 52)))
    for a, q in zip(ins, qps):
        o, p = oracle.ref_intra16_luma_dc(a, q)
        outs.append(o)
        pres.append(p)
    np.savez_compressed(os.path.join(HERE, "dc_transpose.npz"), dc_in=np.array(ins), qp=np.array(qps),
                        dc_out=np.array(outs), pre=np.array(pres))

    # --- SAD (A1/tests/test_cpu_simd_me.c:16-43 + seeded) ---
    a = rng.integers(0, 256, (64, 16, 16), dtype=np.uint8)
    b = rng.integers(0, 256, (64, 16, 16), dtype=np.uint8)
    sads = np.array([oracle.ref_sad16(a[i], b[i]) for i in range(64)], np.uint32)
    np.savez_compressed(os.path.join(HERE, "sad.npz"), a=a, b=b, sad=sads)

    # --- MC, every phase, interior and edges ---
    plane = rng.integers(0, 256, (40, 48), dtype=np.uint8)
    pos, lum = [], []
    for fy in range(4):
        for fx in range(4):
            for (x, y) in ((12, 10), (-3, -2), (40, 30), (0, 0)):
                qx, qy = x * 4 + fx, y * 4 + fy
                pos.append((qx, qy))
                lum.append(oracle.ref_mc_luma(plane, 48, 40, qx, qy))
    uv = rng.integers(0, 256, (20, 48), dtype=np.uint8)
    cpos, chro = [], []
    for pl in range(2):
        for fy in range(8):
            for fx in range(8):
                for (x, y) in ((6, 5), (-2, -1), (20, 16)):
                    ex, ey = x * 8 + fx, y * 8 + fy
                    cpos.append((pl, ex, ey))
                    chro.append(oracle.ref_mc_chroma(uv, 24, 20, pl, ex, ey))
    np.savez_compressed(os.path.join(HERE, "mc.npz"), plane=plane, pos=np.array(pos), luma=np.array(lum), uv=uv,
                        cpos=np.array(cpos), chroma=np.array(chro))

    # --- dequant + inverse + add ---
    blocks, qps, preds, recs = [], [], [], []
    for _ in range(400):
        q = int(rng.integers(0, 52))
        lev = (rng.integers(-12, 13, 16) * (rng.random(16) < 0.4)).astype(np.int16)
        pred = rng.integers(0, 256, (4, 4), dtype=np.uint8)
        dst = pred.copy()
        oracle.ref_idct4_add(dst, lev, q, 0)
        blocks.append(lev)
        qps.append(q)
        preds.append(pred)
        recs.append(dst)
    np.savez_compressed(os.path.join(HERE, "idct.npz"), levels=np.array(blocks), qp=np.array(qps),
                        pred=np.array(preds), rec=np.array(recs))

    # --- deblocking ---
    cases = []
    for ci, (mbw, mbh, qp, intra) in enumerate(((4, 3, 30, 1), (4, 3, 30, 0), (5, 4, 40, 0), (3, 3, 45, 1),
                                                (6, 2, 20, 0), (2, 5, 51, 1))):
        y = np.clip(128 + 30 * rng.standard_normal((mbh * 16, mbw * 16)), 0, 255).astype(np.uint8)
        y = (y // 8 * 8).astype(np.uint8)  # blocky, so filters fire
        uvp = np.clip(128 + 20 * rng.standard_normal((mbh * 8, mbw * 16)), 0, 255).astype(np.uint8)
        nz = (rng.random((mbw * mbh, 24)) < 0.3).astype(np.uint32) * rng.integers(1, 1 << 16, (mbw * mbh, 24)).astype(np.uint32)
        mv = np.zeros((mbw * mbh, 4), np.int32)
        mv[:, :2] = rng.integers(-12, 13, (mbw * mbh, 2))
        yo, uvo = y.copy(), uvp.copy()
        oracle.ref_deblock(mbw, mbh, qp, intra, nz, mv, yo, uvo)
        cases.append(dict(mbw=mbw, mbh=mbh, qp=qp, intra=intra, y=y, uv=uvp, nz=nz, mv=mv, y_out=yo, uv_out=uvo))
    np.savez_compressed(os.path.join(HERE, "deblock.npz"),
                        **{f"c{i}_{k}": v for i, c in enumerate(cases) for k, v in c.items()}, n=len(cases))
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
