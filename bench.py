#!/usr/bin/env python
"""Benchmark of the B200 compute-encoder hot path: 1080p encode fps of the
learned-proposal form against the plain full-search form.

Workload: S concurrent streams (default 8, one context and CUDA stream each)
of 1920x1080 8-bit NV12, IPPP with an IDR every 60 frames, QP 27 (a point of
the 22/27/32/37 sweep), search range 32, lambda 5, spec deblocking on. A step
is one frame of every stream through ME -> P chain (or intra wavefront) ->
deblock. Each stream cycles 60 seeded synthetic frames resident in HBM
(S x 187 MB, far larger than L2). The learned form (value) ranks candidates
with the packaged network - trained in BF16, run in FP8 E4M3 on the tensor
cores - and re-scores the top 4 exactly, falling back to the full search
under the confidence threshold; the first P frame of each GOP has no motion
history and takes the full search. The plain form is the full search on
every P frame. Both are timed in the same run, and again with one stream
(single_stream); the learned form with BF16 inference is timed beside them
(learned_bf16).

  value  learned-form frames/s summed over the S streams and over ranks,
         device-timed with CUDA events (start event on a control stream that
         every context stream waits on, end event after every context stream
         has drained), max over ranks (weak scaling: independent streams per
         GPU, no collective on the data path).
  e2e    the learned form through the reference boundary (per stream
         gpu_compute_upload_nv12 from pinned host memory,
         begin/dispatch/end_picture; then sync_slot and a host read of the
         staged outputs), S streams, double-buffered over the boundary's two
         staging slots (step k+1 is submitted before step k is read back).
  bd_rate the learned form's BD-rate against the plain form (bits from the
         reference's host encoder, CABAC, QP 22/27/32/37, 60 1080p frames),
         measured on a B200 with tests/rd_report.py and recorded in
         profiles/rd_h264_1080p_learned_vs_plain.json.

`--impl reference` times the reference's CPU implementation of the same
frame (the plain form; the reference has no learned form) on the host cores
(oracle/_ref: the reference's AVX2 SAD in the exhaustive search, its C
deblocking filter; the P chain from the CPU restatement), each step a
bounded sample of one frame.
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
    from b200enc import replicas
    return replicas.dist_env()


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
    line = {"metric": "1080p encode fps, learned-proposal form (vs plain full-search form)", "value": round(fps, 4),
            "unit": "frames/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 / fps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32",
            "data": "synthetic (seeded generator, 1080p NV12)", "impl": "reference",
            "config": {"workload": f"{WORKLOAD}_x{args.streams}_streams", "streams_per_gpu": args.streams,
                       "width": W, "height": H, "qp": QP, "search_range": RANGE, "lambda": LAMBDA, "gop": GOP,
                       "deblock": True, "recon_clamp": "coded",
                       "parallelism": "the host's threads on one stream's frames at a time (frames/s does not "
                                      "depend on how many streams share the host)"},
            "cpu_baseline": {"value": round(fps, 4), "unit": "frames/s", "cores": info["cores"],
                             "kind": info["kind"], "sample": info["sample"]},
            "e2e": {"value": round(fps, 4), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU arm

def _frames_pool(seeds, n):
    """Synthetic frames of several streams, generated on the host cores (a
    spawned pool: no CUDA state is forked)."""
    import multiprocessing as mp
    if len(seeds) == 1:
        return [make_frames(seeds[0], n)]
    with mp.get_context("spawn").Pool(min(len(seeds), max(1, (os.cpu_count() or 2) - 1))) as pool:
        return pool.starmap(make_frames, [(s, n) for s in seeds])


def rd_fp8_pct():
    p = os.path.join(ROOT, "profiles", "rd_h264_1080p_learned_fp8_vs_plain.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return round(json.load(f)["bd_rate_learned_fp8_vs_plain_pct"], 3)


def rd_record():
    p = os.path.join(ROOT, "profiles", "rd_h264_1080p_learned_vs_plain.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    fp8 = rd_fp8_pct()
    return {"value_pct": fp8 if fp8 is not None else round(d["bd_rate_learned_vs_plain_pct"], 3),
            "metric": "BD-rate (YUV PSNR) vs plain, learned form with FP8 inference",
            "bf16_pct": round(d["bd_rate_learned_vs_plain_pct"], 3),
            "no_network_pct": round(d["bd_rate_no_network_vs_plain_pct"], 3), "conf": d["conf"],
            "source": "profiles/rd_h264_1080p_learned_fp8_vs_plain.json, profiles/rd_h264_1080p_learned_vs_plain.json "
                      "(tests/rd_report.py on B200)",
            "workload": d["workload"]}


# the headline learned form: FP8 inference (b200enc_ctx_set_me mode 3); mode 1 is BF16 inference
LEARNED = 3


# kernels per frame of each kind (counted from the launch sites)
LAUNCHES = {"i": 2, "p_full": 3, "p_learned": 12}


def run_gpu(args):
    import numpy as np
    import torch
    import b200enc

    from b200enc import replicas

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    os.environ["B200ENC_DEVICE"] = str(local)
    group = replicas.Group("nccl", device="cuda")

    S = args.streams
    host_frames = _frames_pool(replicas.stream_seeds(rank, S), NFRAMES)
    dev = [[b200enc.NV12.from_host(y, uv) for (y, uv) in fr] for fr in host_frames]
    ctxs = []
    for s in range(S):
        c = b200enc.Context()
        c.configure(search_range=RANGE, lam=LAMBDA, zero_thresh=512, coded_clamp=True, deblock=1)
        ctxs.append(c)
    streams = [torch.cuda.ExternalStream(c.stream()) for c in ctxs]
    control = torch.cuda.Stream()

    def barrier():
        group.barrier(torch.cuda.synchronize)

    def max_over_ranks(ms):
        return group.max(ms)

    host_ms = {}

    def arm(mode, nstreams, steps, warmup, perf=False, clocks=False):
        """Encodes warmup + steps frames on each of the first nstreams
        contexts from the start of a GOP; returns (ms, launches, perf, clk)."""
        for c in ctxs[:nstreams]:
            c.set_me(mode, conf=args.conf)
            c.perf(False)
        t = 0

        def one_step(t):
            n = 0
            intra = (t % GOP) == 0
            for s in range(nstreams):
                ctxs[s].encode_device(dev[s][t % NFRAMES], W, H, QP, intra, 1, False)
            if intra:
                n = LAUNCHES["i"]
            elif mode == 0 or (t % GOP) == 1:
                n = LAUNCHES["p_full"]
            else:
                n = LAUNCHES["p_learned"]
            return n * nstreams

        for _ in range(warmup):
            one_step(t)
            t += 1
        barrier()
        if perf:
            ctxs[0].perf(True)
        clk = Clocks(local) if (clocks and rank == 0) else None
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(control)
        for st in streams[:nstreams]:
            st.wait_event(e0)
        launches = 0
        h0 = time.perf_counter()
        for _ in range(steps):
            launches += one_step(t)
            t += 1
        host_issue_s = time.perf_counter() - h0  # host time to enqueue the timed steps
        for st in streams[:nstreams]:
            ev = torch.cuda.Event()
            ev.record(st)
            control.wait_event(ev)
        e1.record(control)
        barrier()
        c = clk.stop() if clk else None
        pf = (ctxs[0].perf_read(False), ctxs[0].perf_read(True)) if perf else None
        host_ms[mode, nstreams] = 1000.0 * host_issue_s / steps
        return max_over_ranks(e0.elapsed_time(e1)), launches, pf, c

    K, Wm = args.steps, args.warmup
    ms_l, launches, _, clk = arm(LEARNED, S, K, Wm, clocks=True)
    ms_p, _, _, _ = arm(0, S, K, Wm)
    ms_b, _, _, _ = arm(1, S, K, Wm)  # the learned form with the network's inference in BF16
    k1 = max(K, 2 * GOP)
    ms_l1, _, perf_l1, _ = arm(LEARNED, 1, k1, Wm, perf=True)
    me_counts = ctxs[0].me_stats()  # the learned form's last P frame
    ms_p1, _, perf_p1, _ = arm(0, 1, k1, Wm, perf=True)
    fps = replicas.aggregate_rate(ws, S * K, ms_l)
    fps_plain = replicas.aggregate_rate(ws, S * K, ms_p)
    fps_bf16 = replicas.aggregate_rate(ws, S * K, ms_b)

    # ---- e2e through the reference boundary, host buffers -----------------
    NP = 30
    pinned = [[(torch.from_numpy(np.ascontiguousarray(y)).pin_memory(),
                torch.from_numpy(np.ascontiguousarray(uv)).pin_memory()) for (y, uv) in fr[:NP]]
              for fr in host_frames]
    imgs = [c.create_image(W, H) for c in ctxs]
    for c in ctxs:
        c.set_me(LEARNED, conf=args.conf)

    # Double-buffered, as the boundary's two staging slots allow: step k+1 is
    # uploaded and submitted before step k's staged results are read, so each
    # stream's copies overlap its (and the other streams') compute. Every
    # step's upload and result read lie inside the timed region.
    def e2e_submit(k):
        slots = []
        for s, c in enumerate(ctxs):
            py, puv = pinned[s][k % NP]
            img, mem = imgs[s]
            rc = c.L.gpu_compute_upload_nv12(b200enc.ctypes.byref(c.ctx), b200enc.ctypes.byref(img), mem,
                                             b200enc.ctypes.c_void_p(py.data_ptr()), W,
                                             b200enc.ctypes.c_void_p(puv.data_ptr()), W, W, H)
            assert rc == 0
            slots.append(c.encode(img, W, H, QP, (k % GOP) == 0, 1, 0, None))
        return slots

    def e2e_collect(slots):
        acc = 0
        for c, slot in zip(ctxs, slots):
            assert c.sync(slot) == 0
            acc += int(c.staging(slot)["nz"][0, 0])  # a host read of each step's result
        return acc

    def e2e_run(k, n):
        pending = None
        for _ in range(n):
            cur = e2e_submit(k)
            if pending is not None:
                e2e_collect(pending)
            pending = cur
            k += 1
        e2e_collect(pending)
        return k

    k = e2e_run(0, Wm)
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(control)
    k = e2e_run(k, K)
    s1.record(control)
    barrier()
    e2e_fps = replicas.aggregate_rate(ws, S * K, max_over_ranks(s0.elapsed_time(s1)))
    for c, (img, mem) in zip(ctxs, imgs):
        c.destroy_image(img, mem)

    if rank == 0:
        peak, peak_kind = measured_peaks()
        pp1, pi1 = perf_l1
        nP = max(1, pp1["frames"])
        stage_ms = {k2: pp1[k2] / nP for k2 in ("me", "chain", "deblock", "staging")}
        plain_stage_ms = {k2: perf_p1[0][k2] / max(1, perf_p1[0]["frames"]) for k2 in ("me", "chain", "deblock")}
        dom = max(("me", "chain", "deblock"), key=lambda k2: stage_ms[k2])
        algo = ALGO_BYTES_PER_MB[dom] * MBS
        ach = algo / (stage_ms[dom] / 1000.0) / 1e9
        tr = traffic_from_profiles(dom)
        pipe_bytes = (ALGO_BYTES_PER_MB["me"] + ALGO_BYTES_PER_MB["chain"] + ALGO_BYTES_PER_MB["deblock"]) * MBS
        line = {
            "metric": "1080p encode fps, learned-proposal form (vs plain full-search form)", "value": round(fps, 2),
            "unit": "frames/s", "n_gpus": ws, "steps": K, "warmup": Wm,
            "ms_per_step": round(ms_l / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8/int32 (integer path), fp8 e4m3 (proposal network inference; trained in bf16)",
            "data": "synthetic (seeded generator: gradients, sigma-8 texture, 6 moving rectangles, pan, noise patch)",
            "config": {"workload": f"{WORKLOAD}_x{S}_streams", "streams_per_gpu": S, "width": W, "height": H,
                       "qp": QP, "search_range": RANGE, "lambda": LAMBDA, "gop": GOP, "deblock": True,
                       "recon_clamp": "coded", "proposal_conf": args.conf,
                       "l2": f"each stream cycles {NFRAMES} resident frames ({S * NFRAMES * W * H * 3 // 2 >> 20} MiB "
                             "> L2)",
                       "parallelism": f"replicas x{ws} (independent streams per GPU)"},
            "plain": {"value": round(fps_plain, 2), "unit": "frames/s", "ms_per_step": round(ms_p / K, 4)},
            "speedup_vs_plain": round(fps / fps_plain, 3),
            "learned_bf16": {"value": round(fps_bf16, 2), "unit": "frames/s", "ms_per_step": round(ms_b / K, 4),
                             "speedup_vs_plain": round(fps_bf16 / fps_plain, 3),
                             "note": "the same learned form with the network's inference in BF16 (set_me mode 1)"},
            "host_issue_ms_per_step": {"learned": round(host_ms[1, S], 4), "plain": round(host_ms[0, S], 4),
                                       "note": "host time to enqueue one step (all streams); compare ms_per_step"},
            "single_stream": {"learned_fps": round(k1 / (ms_l1 / 1000.0), 2),
                              "plain_fps": round(k1 / (ms_p1 / 1000.0), 2),
                              "learned_stage_ms_per_p_frame": {k2: round(v, 4) for k2, v in stage_ms.items()},
                              "plain_stage_ms_per_p_frame": {k2: round(v, 4) for k2, v in plain_stage_ms.items()},
                              "last_p_frame_mbs": dict(zip(("learned", "fallback", "early"), me_counts))},
            "bd_rate": rd_record(),
            "gpu_launches": launches,
            "e2e": {"value": round(e2e_fps, 2), "unit": "frames/s", "h2d_bytes_per_step": S * H2D_PER_STEP,
                    "d2h_bytes_per_step": S * D2H_PER_STEP},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(ach / peak, 5), "peak_kind": peak_kind,
                         "traffic": (round(tr * MBS) if tr is not None else None),
                         "algorithmic_bytes": int(algo),
                         "timing": "single-stream learned run, stage events on the context stream"},
            "hbm_pipeline": {"achieved": round(pipe_bytes * fps / ws / 1e9, 2), "unit": "GB/s",
                             "frac": round(pipe_bytes * fps / ws / 1e9 / peak, 5),
                             "note": "algorithmic bytes of ME + P chain + deblock per P frame x learned-form fps"},
            "clocks": clk,
        }
        if ws == 1 and not args.no_cpu_baseline:
            spf, info = cpu_reference_frame_time(host_frames[0][:2], budget_s=15.0)
            line["cpu_baseline"] = {"value": round(1.0 / spf, 4), "unit": "frames/s", "cores": info["cores"],
                                    "kind": info["kind"], "sample": info["sample"],
                                    "stage_s": {k2: round(v, 4) for k2, v in info["stage_s"].items()}}
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    group.close()


def run_hevc_deblock(args):
    """HEVC deblocking (b200enc_hevc_deblock) on seeded synthetic pictures:
    1080p 8-bit and 2160p 10-bit, enough resident copies to exceed L2, timed
    with CUDA events over `steps` passes; the reference decoder's filter
    (oracle/_ref/libhevcfilt.so) timed on the host threads beside it. Prints
    one JSON line per picture format."""
    import numpy as np
    import torch
    import b200enc
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import hevc_db_inputs as hdi
    hbm_peak, peak_kind = measured_peaks()
    fmts = (("1080p_8bit", dict(seed=11, width=1920, height=1080, bit_depth=8, log2_ctb=6, log2_min_cb=3), 48),
            ("2160p_10bit", dict(seed=16, width=3840, height=2160, bit_depth=10, log2_ctb=6, log2_min_cb=3, slices=4),
             12))
    dev = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()
    for name, kw, npic in fmts:
        case = hdi.make_case(**kw)
        maps = {k: dev(case[k]) for k in ("edges", "mvf", "cbf", "qp_y", "no_filter", "slice_of_ctb", "tile_of_ctb")}
        sfd = dev(case["slice_filter"])
        pics = [[dev(p) for p in case["planes"]] for _ in range(npic)]
        qs = []
        for pl in pics:
            q = hdi.params(b200enc, dict(case, **maps), lambda t: t.data_ptr(), planes=pl, slice_filter=None)
            q.slice_filter, q.n_slice_filter = sfd.data_ptr(), len(case["slice_filter"])
            qs.append(q)
        for q in qs[:args.warmup]:
            b200enc.hevc_deblock(q)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(args.steps):
            b200enc.hevc_deblock(qs[k % npic])
        e1.record()
        torch.cuda.synchronize()
        us = e0.elapsed_time(e1) * 1e3 / args.steps
        bps = 1 if kw["bit_depth"] == 8 else 2
        traffic = 4 * kw["width"] * kw["height"] * 1.5 * bps   # two passes, each reads and writes the picture
        line = {"metric": "HEVC deblocking pictures/s", "workload": name, "value": round(1e6 / us, 1),
                "unit": "pictures/s", "us_per_picture": round(us, 2), "steps": args.steps, "warmup": args.warmup,
                "launches_per_picture": 2, "resident_pictures": npic,
                "roofline": {"bound": "hbm", "achieved": round(traffic / (us * 1e-6) / 1e9, 1),
                             "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s",
                             "frac": round(traffic / (us * 1e-6) / 1e9 / hbm_peak, 4),
                             "traffic_model_bytes": traffic}}
        if not args.no_cpu_baseline and os.path.exists(hdi.FILT_SO):
            t0, n = time.perf_counter(), 0
            while time.perf_counter() - t0 < 3.0:
                hdi.reference(b200enc, case)
                n += 1
            ms = (time.perf_counter() - t0) / n * 1e3
            line["cpu_baseline"] = {"value": round(1e3 / ms, 1), "unit": "pictures/s", "cores": os.cpu_count(),
                                    "kind": "reference", "sample": f"{n} pictures through hevcd_loop_filters"}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--conf", type=float, default=0.9)
    ap.add_argument("--hevc-deblock", action="store_true",
                    help="time b200enc_hevc_deblock instead of the H.264 encode (own JSON lines)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.hevc_deblock:
        run_hevc_deblock(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
