"""RD report of the learned form against the plain full search on the 1080p
workload (seeded synthetic 1920x1080, pan + noise patch, 60 frames IPPP,
R32, CABAC, QP 22/27/32/37): bits, PSNR, BD-rate, fallback counts, for the
network at its default confidence threshold and for the candidate search
without the network. TEST INFRASTRUCTURE (drives the reference encoder in
oracle/_ref).

    python tests/rd_report.py OUT.json [--frames 60] [--weights PATH] [--modes plain,learned_fp8]
"""
import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bc250-vaapi_b200"))

import rd_harness as rh  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--frames", type=int, default=60)
    ap.add_argument("--size", default="1920x1080")
    ap.add_argument("--weights")
    ap.add_argument("--conf", type=float, default=0.9)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--modes", default="plain,learned,no_network",
                    help="comma list of plain, learned, no_network, learned_fp8 (network inference in FP8)")
    a = ap.parse_args()
    import b200enc as gpu
    W, H = (int(v) for v in a.size.split("x"))
    frames = rh.make_frames(W, H, a.frames, seed=a.seed)
    every = {"plain": (rh.PLAIN, 0.0), "learned": (rh.LEARNED, a.conf), "no_network": (rh.CANDIDATES, -1.0),
             "learned_fp8": (rh.LEARNED_FP8, a.conf)}
    runs = {m: every[m] for m in a.modes.split(",")}
    res = {}
    for name, (mode, conf) in runs.items():
        res[name] = [rh.encode(gpu, frames, W, H, qp, mode, conf, a.weights) for qp in (22, 27, 32, 37)]
        for r in res[name]:
            r.pop("frame_bits")
    rep = {"workload": f"{W}x{H} synthetic pan+noise, {a.frames} frames IPPP GOP60, R32 lambda5, CABAC, QP 22/27/32/37",
           "conf": a.conf, "runs": res}
    for m in ("learned", "no_network", "learned_fp8"):
        if m in res and "plain" in res:
            rep[f"bd_rate_{m}_vs_plain_pct"] = rh.bd_rate(res["plain"], res[m])
            rep[f"bd_rate_{m}_vs_plain_y_pct"] = rh.bd_rate(res["plain"], res[m], "psnr_y")
    with open(a.out, "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps({k: v for k, v in rep.items() if k != "runs"}, indent=1))


if __name__ == "__main__":
    main()
