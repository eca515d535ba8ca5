#!/usr/bin/env python
"""Benchmark of the B200 compute-encoder hot path: 1080p encode fps.

Workload (plain full-search form): 1920x1080 8-bit NV12, IPPP with an IDR
every 60 frames, QP 27 (a point of the 22/27/32/37 sweep), integer full
search over [-32,32]^2 + half/quarter-pel refine, spec deblocking on. A step
is one frame through ME -> P chain (or intra wavefront) -> deblock. Inputs
are 60 seeded synthetic frames resident in HBM (187 MB, larger than L2), so
every step reads a frame that is not in L2.

  value  frames/s over K timed steps, device-timed with CUDA events on the
         library's stream, max over ranks, summed over ranks (weak scaling:
         one independent stream per GPU, no collective on the data path).
  e2e    the same through the reference boundary (gpu_compute_upload_nv12
         from pinned host memory, begin/dispatch/end_picture, sync_slot and
         the staging read-back of levels/dc/nz/pred_mode/mv every step).

`--impl reference` times the reference's CPU implementation of the same
frame on the host cores (oracle/_ref: the reference's AVX2 SAD in the
exhaustive search, its C deblocking filter; the P chain from the CPU
restatement), each step a bounded sample of one frame.
"""
import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "bc250-vaapi_b200"))

W, H, QP, RANGE, LAMBDA, GOP, NFRAMES = 1920, 1080, 27, 32, 5, 60, 60
MBW, MBH = (W + 15) // 16, (H + 15) // 16
MBS = MBW * MBH
WORKLOAD = "h264_1080p_ippp_fullsearch_r32"
# Algorithmic bytes per macroblock of each stage (per launch = x MBS):
#   ME: current + reference luma once (2 B/px) + the 16-byte MV
#   P chain: src YUV 1.5 + ref YUV 1.5 + levels 3.0 + nz 0.375 + dc 0.375 + recon 1.5 B/px
#   deblock: recon read+write 3.0 + nz 0.375 + MV 0.0625 B/px
ALGO_BYTES_PER_MB = {"me": 2 * 256 + 16, "chain": 8.25 * 256, "deblock": 3.4375 * 256}
H2D_PER_STEP = W * H * 3 // 2
D2H_PER_STEP = MBS * (768 + 96 + 4 + 16 + 96) + 8


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "20", "-i", str(gpu_index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def traffic_from_profiles(stage):
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(stage)
    return None if v is None else float(v)


def make_frames(seed_stream, n):
    from b200enc import synth
    seq = synth.workload("h264_1080p", seed=0, stream=seed_stream)
    return [seq.frame(t) for t in range(n)]


# ----------------------------------------------------------------- CPU arm

def cpu_reference_frame_time(frames, budget_s=15.0, threads=None):
    """Seconds one 1080p P frame takes on the host cores through the
    reference's CPU code, measured on a bounded sample and scaled by the
    macroblock rows processed. Returns (seconds_per_frame, info)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    threads = threads or os.cpu_count()
    (y0, uv0), (y1, uv1) = frames[0], frames[1]
    CW, CH = MBW * 16, MBH * 16
    ry = np.pad(y0, ((0, CH - H), (0, 0)), mode="edge")
    ruv = np.pad(uv0, ((0, CH // 2 - H // 2), (0, 0)), mode="edge")
    kind = "reference" if oracle.ref_available() else "port"
    # ME integer search: rows sampled until ~half the budget is spent
    t0 = time.perf_counter()
    rows = 0
    while rows < MBH and time.perf_counter() - t0 < budget_s * 0.5:
        r0 = rows
        r1 = min(MBH, rows + max(1, threads // 4))
        if kind == "reference":
            oracle.ref_full_search_int(y1, W, H, ry, CW, CH, RANGE, LAMBDA, r0, r1, threads)
        else:
            f = oracle.frame(W, 16 * (r1 - r0), QP)
            oracle.me_frame(f, np.ascontiguousarray(y1[16 * r0:16 * r1]), ry, RANGE, LAMBDA)
        rows = r1
    t_me = (time.perf_counter() - t0) / rows * MBH
    # P chain (CPU restatement, one thread) and deblocking over the full frame
    f = oracle.frame(W, H, QP)
    mv = np.zeros((MBS, 4), np.int32)
    rec_y = np.zeros((CH, CW), np.uint8)
    rec_uv = np.zeros((CH // 2, CW), np.uint8)
    t1 = time.perf_counter()
    o = oracle.p_frame(f, y1, uv1, ry, ruv, mv, rec_y, rec_uv)
    t_chain = time.perf_counter() - t1
    t2 = time.perf_counter()
    if kind == "reference":
        oracle.ref_deblock(MBW, MBH, QP, 0, o["nz"], o["mv"], rec_y, rec_uv)
    else:
        oracle.deblock(MBW, MBH, QP, 0, o["nz"], o["mv"], rec_y, rec_uv)
    t_db = time.perf_counter() - t2
    sample = (f"one 1080p P frame: full search +-{RANGE} on {rows}/{MBH} MB rows "
              f"({'reference cpu_simd_sad_16x16 AVX2' if kind == 'reference' else 'CPU restatement'}, "
              f"{threads} threads) scaled to {MBH} rows; P chain (CPU restatement, 1 thread) and "
              f"{'reference h264d_deblock_picture' if kind == 'reference' else 'restated deblocking'} (1 thread) "
              f"on the whole frame")
    return t_me + t_chain + t_db, dict(kind=kind, cores=threads, sample=sample,
                                       stage_s=dict(me=t_me, chain=t_chain, deblock=t_db))


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    frames = make_frames(0, 2)
    budget = max(0.25, min(15.0, 120.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_reference_frame_time(frames, budget_s=budget / 4)
    times = []
    info = None
    for _ in range(args.steps):
        t, info = cpu_reference_frame_time(frames, budget_s=budget)
        times.append(t)
    fps = len(times) / sum(times)
    line = {"metric": "1080p encode fps (plain full-search form)", "value": round(fps, 4), "unit": "frames/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 / fps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32",
            "data": "synthetic (seeded generator, 1080p NV12)", "impl": "reference",
            "config": {"workload": WORKLOAD, "width": W, "height": H, "qp": QP, "search_range": RANGE,
                       "gop": GOP, "deblock": True},
            "cpu_baseline": {"value": round(fps, 4), "unit": "frames/s", "cores": info["cores"],
                             "kind": info["kind"], "sample": info["sample"]},
            "e2e": {"value": round(fps, 4), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU arm

def run_gpu(args):
    import numpy as np
    import torch
    import b200enc

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    os.environ["B200ENC_DEVICE"] = str(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist

    frames = make_frames(rank, NFRAMES)
    dev = [b200enc.NV12.from_host(y, uv) for (y, uv) in frames]
    ctx = b200enc.Context()
    ctx.configure(search_range=RANGE, lam=LAMBDA, zero_thresh=512, coded_clamp=True, deblock=1)
    stream = torch.cuda.ExternalStream(ctx.stream())

    def step(t, stage=False):
        ctx.encode_device(dev[t % NFRAMES], W, H, QP, (t % GOP) == 0, 1, stage)

    t = 0
    for _ in range(args.warmup):
        step(t)
        t += 1
    torch.cuda.synchronize()
    ctx.perf(True)

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    clocks = Clocks(local) if rank == 0 else None
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    for _ in range(args.steps):
        launches += 2 if (t % GOP) == 0 else 3
        step(t)
        t += 1
    e1.record(stream)
    barrier()
    clk = clocks.stop() if clocks else None
    ms = e0.elapsed_time(e1)
    if pg:
        tt = torch.tensor([ms], device="cuda")
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        ms = float(tt.item())
    fps = ws * args.steps / (ms / 1000.0)
    perf_p = ctx.perf_read(False)
    perf_i = ctx.perf_read(True)

    # searched macroblocks of the last P frame (zero-MV early-outs do no search)
    out = {}
    ok = ctx.L.b200enc_ctx_device_outputs(b200enc.ctypes.byref(ctx.ctx), None, None, None, None,
                                          b200enc.ctypes.byref(mvp := b200enc.ctypes.c_void_p()))
    mvh = b200enc.device_view(mvp.value, MBS * 16).cpu().numpy().view(np.int32).reshape(MBS, 4)
    searched = int(np.sum(~((mvh[:, 0] == 0) & (mvh[:, 1] == 0) & (mvh[:, 2].view(np.uint32) <= 512))))

    # ---- e2e through the reference boundary, host buffers -----------------
    pinned = []
    for (y, uv) in frames[:8]:
        py = torch.from_numpy(np.ascontiguousarray(y)).pin_memory()
        puv = torch.from_numpy(np.ascontiguousarray(uv)).pin_memory()
        pinned.append((py, puv))
    img, mem = ctx.create_image(W, H)
    L, c = ctx.L, b200enc.ctypes.byref(ctx.ctx)

    def e2e_step(k):
        py, puv = pinned[k % len(pinned)]
        rc = L.gpu_compute_upload_nv12(c, b200enc.ctypes.byref(img), mem, b200enc.ctypes.c_void_p(py.data_ptr()), W,
                                       b200enc.ctypes.c_void_p(puv.data_ptr()), W, W, H)
        assert rc == 0
        slot = ctx.encode(img, W, H, QP, (k % GOP) == 0, 1, 0, None)
        assert ctx.sync(slot) == 0
        st = ctx.staging(slot)
        return int(st["nz"][0, 0])  # a read of the step's result on the host

    for k in range(args.warmup):
        e2e_step(k)
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for k in range(args.steps):
        e2e_step(k + 1)
    s1.record(stream)
    barrier()
    ems = s0.elapsed_time(s1)
    if pg:
        tt = torch.tensor([ems], device="cuda")
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        ems = float(tt.item())
    e2e_fps = ws * args.steps / (ems / 1000.0)
    ctx.destroy_image(img, mem)

    if rank == 0:
        peak, peak_kind = measured_peaks()
        nP = max(1, perf_p["frames"])
        stage_ms = {k: perf_p[k] / nP for k in ("me", "chain", "deblock", "staging")}
        dom = max(("me", "chain", "deblock"), key=lambda k: stage_ms[k])
        algo = ALGO_BYTES_PER_MB[dom] * MBS
        ach = algo / (stage_ms[dom] / 1000.0) / 1e9
        tr = traffic_from_profiles(dom)
        me_ops = searched * ((2 * RANGE + 1) ** 2 * 256 + 16 * 256)
        line = {
            "metric": "1080p encode fps (plain full-search form)", "value": round(fps, 3), "unit": "frames/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32",
            "data": "synthetic (seeded generator: gradients, sigma-8 texture, 6 moving rectangles, pan, noise patch)",
            "config": {"workload": WORKLOAD, "width": W, "height": H, "qp": QP, "search_range": RANGE,
                       "lambda": LAMBDA, "gop": GOP, "deblock": True, "recon_clamp": "coded",
                       "l2": f"inputs cycle through {NFRAMES} resident frames ({NFRAMES * W * H * 3 // 2 >> 20} MiB > L2)",
                       "parallelism": f"replicas x{ws} (one stream per GPU)"},
            "gpu_launches": launches,
            "e2e": {"value": round(e2e_fps, 3), "unit": "frames/s", "h2d_bytes_per_step": H2D_PER_STEP,
                    "d2h_bytes_per_step": D2H_PER_STEP},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(ach / peak, 5), "peak_kind": peak_kind,
                         "traffic": (round(tr * MBS) if tr is not None else None),
                         "algorithmic_bytes": int(algo)},
            "stages_ms_per_p_frame": {k: round(v, 4) for k, v in stage_ms.items()},
            "stages_ms_per_i_frame": ({k: round(perf_i[k] / perf_i["frames"], 4) for k in ("chain", "deblock")}
                                      if perf_i["frames"] else None),
            "me_int": {"searched_mbs": searched, "abs_diff_per_s": round(me_ops / (stage_ms["me"] / 1000.0), 1)},
            "clocks": clk,
        }
        if ws == 1 and not args.no_cpu_baseline:
            spf, info = cpu_reference_frame_time(frames[:2], budget_s=15.0)
            line["cpu_baseline"] = {"value": round(1.0 / spf, 4), "unit": "frames/s", "cores": info["cores"],
                                    "kind": info["kind"], "sample": info["sample"],
                                    "stage_s": {k: round(v, 4) for k, v in info["stage_s"].items()}}
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
