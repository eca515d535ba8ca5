#!/usr/bin/env python
"""Benchmark of the B200 compute-encoder hot path: 1080p encode fps of the
learned-proposal form against the plain full-search form.

Workload: S concurrent streams (default 8, one context and CUDA stream each)
of 1920x1080 8-bit NV12, IPPP with an IDR every 60 frames, QP 27 (a point of
the 22/27/32/37 sweep), search range 32, lambda 5, spec deblocking on. Stream
s runs its GOP s*60/S frames ahead of stream 0, as independent encoders do,
so every timed window holds I frames at the GOP's rate (one per stream per 60
frames) whatever the step count. A step is one frame of every stream through
ME -> P chain (or intra wavefront) -> deblock. Each stream cycles 60 seeded
synthetic frames resident in HBM (S x 187 MB, far larger than L2). The
learned form (value) ranks candidates with the packaged network - trained in
BF16, run in FP8 E4M3 on the tensor cores - and re-scores the top 4 exactly,
falling back to the full search under the confidence threshold; the first P
frame after each IDR has no motion history and takes the full search. The
plain form is the full search on every P frame. Both are timed in the same
run, and again with one stream (single_stream); the learned form with BF16
inference is timed beside them (learned_bf16).

  value  learned-form frames/s summed over the S streams and over ranks,
         device-timed with CUDA events (start event on a control stream that
         every context stream waits on, end event after every context stream
         has drained), max over ranks (weak scaling: independent streams per
         GPU, no collective on the data path).
  e2e    the learned form through the reference boundary with the
         bitstream as the result: per stream gpu_compute_upload_nv12 from
         pinned host memory, begin/dispatch/end_picture with GPU entropy
         coding (b200enc_ctx_set_entropy mode 2: CAVLC slice data written by
         the GPU into mapped host memory), then b200enc_ctx_slice_nals
         assembling the frame's Annex B slice NAL units on the host (one
         thread per stream); S streams, double-buffered over the boundary's
         two slots (step k+1 is submitted before step k is collected).
  e2e_staging  the same boundary with the staged outputs as the result
         (sync_slot and a host read of the levels, DC, nz, modes, vectors the
         reference's host entropy coder consumes).
  full_encode  the rate an application sees: S streams, one host thread
         each, through the reference's unchanged host encoder
         (h264_encoder_encode_frame_ext in oracle/_ref/libh264enc_b200.so:
         upload, the GPU hot path, CAVLC or CABAC slices on the host cores),
         wall clock over the timed frames.
  me_int the plain full search's integer rate (abs-diffs/s) on one stream.
  bd_rate the learned form's BD-rate against the plain form (bits from the
         reference's host encoder, CABAC, QP 22/27/32/37, 60 1080p frames),
         measured on a B200 with tests/rd_report.py and recorded in
         profiles/rd_h264_1080p_learned_fp8_vs_plain.json.

`--impl reference` times the reference's CPU implementation of the same
frames (the plain form; the reference has no learned form) on the host cores
(oracle/_ref: the reference's AVX2 SAD in the exhaustive search, its C
deblocking filter; the P chain with the frame's own full-search MVs and the
I frame from the CPU restatement), each step a bounded sample of a GOP's
frame mix.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "bc250-vaapi_b200"))

W, H, QP, RANGE, LAMBDA, GOP, NFRAMES = 1920, 1080, 27, 32, 5, 60, 60
MBW, MBH = (W + 15) // 16, (H + 15) // 16
MBS = MBW * MBH
WORKLOAD = "h264_1080p_ippp_fullsearch_r32"
METRIC = "1080p encode fps, learned-proposal form (vs plain full-search form)"
# Algorithmic bytes per macroblock of each stage (per launch = x MBS):
#   ME: current + reference luma once (2 B/px) + the 16-byte MV
#   P chain: src YUV 1.5 + ref YUV 1.5 + levels 3.0 + nz 0.375 + dc 0.375 + recon 1.5 B/px
#   intra: the P chain's bytes without the reference (6.75 B/px)
#   deblock: recon read+write 3.0 + nz 0.375 + MV 0.0625 B/px
ALGO_BYTES_PER_MB = {"me": 2 * 256 + 16, "chain": 8.25 * 256, "intra": 6.75 * 256, "deblock": 3.4375 * 256}
# Integer ME work per searched MB: (2R+1)^2 candidates x 256 abs-diffs + 16 sub-pel candidates x 256
ME_ABSDIFF_PER_MB = (2 * RANGE + 1) ** 2 * 256 + 16 * 256
H2D_PER_STEP = W * H * 3 // 2
D2H_PER_STEP = MBS * (768 + 96 + 4 + 16 + 96) + 8
ENC_SO = os.path.join(ROOT, "oracle", "_ref", "libh264enc_b200.so")


def dist_env():
    from b200enc import replicas
    return replicas.dist_env()


def gop_phase(s, S):
    """GOP offset of stream s among S: the streams' IDRs are spread evenly."""
    return (s * GOP) // max(1, S)


def bench_config(S, conf):
    """The workload's configuration, printed identically by both arms."""
    return {"workload": f"{WORKLOAD}_x{S}_streams", "streams_per_gpu": S, "width": W, "height": H, "qp": QP,
            "search_range": RANGE, "lambda": LAMBDA, "gop": GOP, "gop_phase": "stream s: s*gop/streams",
            "deblock": True, "recon_clamp": "coded", "proposal_conf": conf,
            "l2": f"each stream cycles {NFRAMES} resident frames ({S * NFRAMES * W * H * 3 // 2 >> 20} MiB > L2)",
            "parallelism": "independent streams (one context each); replicas across GPUs"}


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
    """Seconds one 1080p frame of the GOP's mix (59 P frames, 1 I frame)
    takes on the host cores through the reference's CPU code. The P frame's
    full search is timed on a bounded sample of macroblock rows and scaled;
    its P chain runs with the frame's own full-search MVs (every sub-pel
    phase the search picks), macroblocks in parallel; deblocking is the
    reference's filter as shipped (one thread); the I frame is the
    restatement's intra wavefront in raster order (one thread: its
    macroblocks depend on one another). Returns (seconds_per_frame, info)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    threads = threads or os.cpu_count()
    oracle.set_threads(threads)
    (y0, uv0), (y1, uv1) = frames[0], frames[1]
    CW, CH = MBW * 16, MBH * 16
    kind = "reference" if oracle.ref_available() else "port"
    f = oracle.frame(W, H, QP)
    # the reference picture: frame 0 intra-coded and deblocked
    ry = np.zeros((CH, CW), np.uint8)
    ruv = np.zeros((CH // 2, CW), np.uint8)
    t0 = time.perf_counter()
    oi = oracle.i_frame(f, y0, uv0, ry, ruv)
    t_intra = time.perf_counter() - t0
    t0 = time.perf_counter()
    if kind == "reference":
        oracle.ref_deblock(MBW, MBH, QP, 1, oi["nz"], oi["mv"], ry, ruv)
    else:
        oracle.deblock(MBW, MBH, QP, 1, oi["nz"], oi["mv"], ry, ruv)
    t_db_i = time.perf_counter() - t0
    # ME integer search: rows sampled until ~half the budget is spent
    t0 = time.perf_counter()
    rows = 0
    while rows < MBH and time.perf_counter() - t0 < budget_s * 0.5:
        r0 = rows
        r1 = min(MBH, rows + max(1, threads // 4))
        if kind == "reference":
            oracle.ref_full_search_int(y1, W, H, ry, CW, CH, RANGE, LAMBDA, r0, r1, threads)
        else:
            fr = oracle.frame(W, 16 * (r1 - r0), QP)
            oracle.me_frame(fr, np.ascontiguousarray(y1[16 * r0:16 * r1]), ry[16 * r0:], RANGE, LAMBDA)
        rows = r1
    t_me = (time.perf_counter() - t0) / rows * MBH
    # the frame's own MVs (full search + sub-pel refine), not timed here
    mv = oracle.me_frame(f, y1, ry, RANGE, LAMBDA)
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
    t_p = t_me + t_chain + t_db
    t_i = t_intra + t_db_i
    sample = (f"1080p GOP mix (59 P + 1 I per 60 frames). P frame: full search +-{RANGE} on {rows}/{MBH} MB rows "
              f"({'reference cpu_simd_sad_16x16 AVX2' if kind == 'reference' else 'CPU restatement'}, "
              f"{threads} threads) scaled to {MBH} rows; P chain (CPU restatement, {threads} threads, the frame's "
              f"own full-search MVs); {'reference h264d_deblock_picture' if kind == 'reference' else 'restated deblocking'}"
              f" (1 thread). I frame: intra wavefront restatement (1 thread) + the same deblocking")
    return ((GOP - 1) * t_p + t_i) / GOP, dict(kind=kind, cores=threads, sample=sample,
                                               stage_s=dict(me=t_me, chain=t_chain, deblock=t_db, intra=t_intra,
                                                            deblock_intra=t_db_i))


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
    line = {"metric": METRIC, "value": round(fps, 4), "unit": "frames/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 / fps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32",
            "data": "synthetic (seeded generator: gradients, sigma-8 texture, 6 moving rectangles, pan, noise patch)",
            "impl": "reference", "config": bench_config(args.streams, args.conf),
            "cpu_baseline": {"value": round(fps, 4), "unit": "frames/s", "cores": info["cores"],
                             "kind": info["kind"], "sample": info["sample"],
                             "parallelism": "the host's threads on one stream's frames at a time (frames/s does not "
                                            "depend on how many streams share the host)",
                             "stage_s": {k: round(v, 4) for k, v in info["stage_s"].items()}},
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


class GopSchedule:
    """Frame kinds of S streams with spread GOP phases. Each arm starts every
    stream with an IDR (a warm-up step), then stream s follows its phase:
    intra when (t + phase_s) % GOP == 0. A P frame is learned when its stream
    has a P frame since the last IDR (the motion history the candidates come
    from)."""

    def __init__(self, S):
        self.S = S
        self.phase = [gop_phase(s, S) for s in range(S)]
        self.since_i = [0] * S

    def kind(self, s, t, learned):
        """'i', 'p_full' or 'p_learned' for stream s at step t (advances)."""
        if t == 0 or (t + self.phase[s]) % GOP == 0:
            self.since_i[s] = 0
            return "i"
        self.since_i[s] += 1
        return "p_learned" if (learned and self.since_i[s] >= 2) else "p_full"


def slice_header_bits(first_mb, idr, frame_num, poc, idr_pic_id=0):
    """A CAVLC slice header in the reference's layout (encoder_h264.c:3093-3126:
    log2_max_frame_num 8, POC type 0 with 8 LSBs, slice QP at the PPS's,
    deblocking on) as (16 header bytes MSB first, bit count)."""
    bits = []

    def ue(v):
        c = v + 1
        n = c.bit_length()
        bits.append("0" * (n - 1) + format(c, "b"))

    ue(first_mb)
    ue(7 if idr else 5)
    ue(0)
    bits.append(format(frame_num & 255, "08b"))
    if idr:
        ue(idr_pic_id)
    bits.append(format(poc & 255, "08b"))
    bits.append("000" if not idr else "00")
    bits.append("1")  # slice_qp_delta 0
    bits.append("1")  # disable_deblocking_filter_idc 0
    bits.append("11")  # alpha / beta offsets 0
    b = "".join(bits)
    return int(b, 2) << (128 - len(b)), len(b)


def e2e_entropy(ctxs, imgs, pinned, esched, S, steps, warmup, control, barrier, max_over_ranks, ws):
    """Frames/s of the whole bitstream path through the boundary with GPU
    entropy coding (b200enc_ctx_set_entropy mode 2): pinned upload, the GPU
    stages, CAVLC slice data on the GPU written into the slot's mapped host
    memory, and the Annex B slice NAL units assembled on the host
    (b200enc_ctx_slice_nals: slice headers, emulation prevention) by one
    host thread per stream. Double-buffered like the e2e figure; device time
    between two events on the control stream, every step's upload and
    bitstream assembly inside it. Returns (frames/s, Mbit per frame)."""
    import concurrent.futures as cf
    import numpy as np
    import torch
    import b200enc
    from b200enc import replicas
    NS = 4
    NP = len(pinned[0])
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    for c in ctxs:
        c.set_entropy(2)
    heads = {}
    for idr in (0, 1):
        h = np.zeros((NS, 16), np.uint8)
        hb = np.zeros(NS, np.int32)
        for k in range(NS):
            v, n = slice_header_bits(k * mbs // NS, bool(idr), 0 if idr else 1, 0 if idr else 2)
            h[k] = np.frombuffer(v.to_bytes(16, "big"), np.uint8)
            hb[k] = n
        heads[idr] = (h, hb)
    outs = [np.zeros(mbs * 2600, np.uint8) for _ in range(S)]
    nbytes = [0] * S
    pool = cf.ThreadPoolExecutor(max_workers=S)

    def submit(k):
        slots = []
        for s, c in enumerate(ctxs):
            py, puv = pinned[s][k % NP]
            img, mem = imgs[s]
            rc = c.L.gpu_compute_upload_nv12(b200enc.ctypes.byref(c.ctx), b200enc.ctypes.byref(img), mem,
                                             b200enc.ctypes.c_void_p(py.data_ptr()), W,
                                             b200enc.ctypes.c_void_p(puv.data_ptr()), W, W, H)
            assert rc == 0
            idr = esched.kind(s, k, True) == "i"
            slots.append((c.encode(img, W, H, QP, idr, NS, 0, None), idr))
        return slots

    def collect_one(s, slot, idr):
        h, hb = heads[int(idr)]
        n = ctxs[s].slice_nals(slot, h, hb, 3 if idr else 2, 5 if idr else 1, outs[s])
        nbytes[s] += n

    def collect(slots):
        list(pool.map(lambda a: collect_one(a[0], *a[1]), enumerate(slots)))

    def run(k, n):
        pending = None
        for _ in range(n):
            cur = submit(k)
            if pending is not None:
                collect(pending)
            pending = cur
            k += 1
        collect(pending)
        return k

    k = run(0, warmup)
    for s in range(S):
        nbytes[s] = 0
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(control)
    run(k, steps)
    e1.record(control)
    barrier()
    pool.shutdown()
    for c in ctxs:
        c.set_entropy(0)
    fps = replicas.aggregate_rate(ws, S * steps, max_over_ranks(e0.elapsed_time(e1)))
    return fps, 8.0 * sum(nbytes) / (S * steps) / 1e6


def full_encode(args, host_frames, S, steps, warmup, profile, me):
    """Frames/s of S streams through the reference's host encoder
    (h264_encoder_encode_frame_ext), one host thread per stream: pinned
    upload, the GPU hot path, the host's CAVLC (profile 66) or CABAC (77)
    slices. Wall clock over `steps` frames per stream, all streams at once;
    stream s first encodes gop_phase(s) + warmup frames so the IDRs spread."""
    import ctypes
    import numpy as np
    import torch
    import b200enc
    if not os.path.exists(ENC_SO):
        return {"unavailable": "oracle/_ref/libh264enc_b200.so not built"}
    os.environ.update({"BC250_FORCE_QP": str(QP), "BC250_FORCE_TIER": "0", "BC250_SLICES_PER_FRAME": "4",
                       "BC250_FORCE_SLICES": "0", "BC250_THREADS": "4", "B200ENC_SEARCH_RANGE": str(RANGE),
                       "B200ENC_ME": me})
    enc = ctypes.CDLL(ENC_SO)
    L = b200enc.lib()
    enc.h264_encoder_create.restype = ctypes.c_void_p
    enc.h264_encoder_create.argtypes = [ctypes.POINTER(b200enc.GpuContext), ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
    enc.h264_encoder_encode_frame_ext.argtypes = [ctypes.c_void_p, ctypes.POINTER(b200enc.GpuContext),
                                                  b200enc.GpuImage, b200enc.GpuMemory, ctypes.c_void_p,
                                                  ctypes.c_size_t]
    NP = 30
    pinned = [[(torch.from_numpy(np.ascontiguousarray(y)).pin_memory(),
                torch.from_numpy(np.ascontiguousarray(uv)).pin_memory()) for (y, uv) in fr[:NP]]
              for fr in host_frames[:S]]
    ctxs, encs, imgs, outs = [], [], [], []
    for s in range(S):
        c = b200enc.GpuContext()
        assert enc.bc250_gpu_init(ctypes.byref(c)) == 0
        e = enc.h264_encoder_create(ctypes.byref(c), W, H, 30, 8_000_000, profile)
        assert e
        enc.h264_encoder_set_gop_size(ctypes.c_void_p(e), ctypes.c_uint32(GOP))
        img, mem = b200enc.GpuImage(), b200enc.GpuMemory()
        assert L.gpu_compute_create_image(ctypes.byref(c), W, H, 0, ctypes.byref(img), ctypes.byref(mem)) == 0
        ctxs.append(c)
        encs.append(e)
        imgs.append((img, mem))
        outs.append(np.zeros(W * H * 4, np.uint8))
    bits = [0] * S
    errors = []
    gate = threading.Barrier(S + 1)

    def one(s, k):
        py, puv = pinned[s][k % NP]
        img, mem = imgs[s]
        c = ctypes.byref(ctxs[s])
        if L.gpu_compute_upload_nv12(c, ctypes.byref(img), mem, ctypes.c_void_p(py.data_ptr()), W,
                                     ctypes.c_void_p(puv.data_ptr()), W, W, H) != 0:
            raise RuntimeError("upload failed")
        n = enc.h264_encoder_encode_frame_ext(ctypes.c_void_p(encs[s]), c, img, mem,
                                              ctypes.c_void_p(outs[s].ctypes.data), outs[s].nbytes)
        if n <= 0:
            raise RuntimeError(f"encoder returned {n}")
        return n

    def worker(s):
        try:
            k = 0
            for _ in range(gop_phase(s, S) + warmup):
                one(s, k)
                k += 1
            gate.wait()
            for _ in range(steps):
                bits[s] += 8 * one(s, k)
                k += 1
            gate.wait()
        except Exception as exc:  # noqa: BLE001 - reported in the JSON line
            errors.append(repr(exc))
            gate.abort()

    th = [threading.Thread(target=worker, args=(s,)) for s in range(S)]
    for t in th:
        t.start()
    try:
        gate.wait()
        t0 = time.perf_counter()
        gate.wait()
        wall = time.perf_counter() - t0
    except threading.BrokenBarrierError:
        wall = None
    for t in th:
        t.join()
    for s in range(S):
        enc.h264_encoder_destroy(ctypes.c_void_p(encs[s]))
        L.gpu_compute_destroy_image(ctypes.byref(ctxs[s]), *imgs[s])
        L.bc250_gpu_destroy(ctypes.byref(ctxs[s]))
    for k in ("B200ENC_ME", "B200ENC_SEARCH_RANGE"):
        os.environ.pop(k, None)
    if errors or not wall:
        return {"unavailable": "; ".join(errors) or "no timing"}
    return {"value": round(S * steps / wall, 2), "unit": "frames/s", "streams": S, "frames_per_stream": steps,
            "entropy": "CAVLC" if profile == 66 else "CABAC", "slices_per_frame": 4, "host_threads_per_stream": 4,
            "host_cores": os.cpu_count(), "mbit_per_frame": round(sum(bits) / (S * steps) / 1e6, 4),
            "timing": "wall clock, upload + encode_frame_ext per frame, all streams in parallel threads"}


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
    frame_kinds = {}

    def arm(mode, nstreams, steps, warmup, perf=False, clocks=False):
        """Encodes warmup + steps frames on each of the first nstreams
        contexts (the first warm-up step an IDR on every stream, then the
        streams' GOP phases); returns (ms, launches, perf, clk)."""
        for c in ctxs[:nstreams]:
            c.set_me(mode, conf=args.conf)
            c.perf(False)
        sched = GopSchedule(nstreams)
        kinds = {"i": 0, "p_full": 0, "p_learned": 0}

        def one_step(t, count):
            n = 0
            for s in range(nstreams):
                k = sched.kind(s, t, mode != 0)
                ctxs[s].encode_device(dev[s][t % NFRAMES], W, H, QP, k == "i", 1, False)
                n += LAUNCHES[k]
                if count:
                    kinds[k] += 1
            return n

        t = 0
        for _ in range(warmup):
            one_step(t, False)
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
            launches += one_step(t, True)
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
        frame_kinds[mode, nstreams] = kinds
        return max_over_ranks(e0.elapsed_time(e1)), launches, pf, c

    K, Wm = args.steps, args.warmup
    if args.profile_arm:
        # one arm only, for a profiler's launch list; no JSON line
        mode = {"learned": LEARNED, "plain": 0, "learned_bf16": 1}[args.profile_arm]
        arm(mode, S, K, Wm)
        for c in ctxs:
            c.close()
        group.close()
        return
    from b200enc import autotune
    tuned = {}

    def tune_arm(mode):
        """Launch parameters of one form, picked by the autotuner for this
        workload's throughput (8 streams, 24 steps per score, median of 3);
        both forms get their own."""
        if args.no_tune:
            autotune.apply({k2: 0 for k2 in autotune.KEYS})
            return {k2: 0 for k2 in autotune.KEYS}
        names = [n for n in autotune.TUNED
                 if mode != 0 or n not in ("rescore_ctas_per_sm", "fallback_ctas_per_sm")]
        t0 = time.perf_counter()
        vals, scores = autotune.tune_throughput(lambda: arm(mode, S, 24, 3)[0], MBH, names, reps=3)
        tuned["learned" if mode else "plain"] = {
            "values": {n: vals[n] for n in names}, "seconds": round(time.perf_counter() - t0, 2),
            "ms_per_24_steps": {n: {str(v): round(t, 3) for v, t in sc.items()} for n, sc in scores.items()}}
        return vals

    k1 = max(K, 2 * GOP)

    def one_stream(mode, vals):
        """The single-stream arm: the tuned values but the built-in deblocking
        tile (8 x 8, the latency choice; the throughput choice is wider)."""
        autotune.apply(dict(vals, deblock_tile_w=0, deblock_tile_h=0))
        r = arm(mode, 1, k1, Wm, perf=True)
        autotune.apply(vals)
        return r

    vals_l = tune_arm(LEARNED)
    ms_l, launches, _, clk = arm(LEARNED, S, K, Wm, clocks=True)
    ms_b, _, _, _ = arm(1, S, K, Wm)  # the learned form with the network's inference in BF16
    ms_l1, _, perf_l1, _ = one_stream(LEARNED, vals_l)
    me_counts = ctxs[0].me_stats()  # the learned form's last P frame
    vals_p = tune_arm(0)
    ms_p, _, _, _ = arm(0, S, K, Wm)
    ms_p1, _, perf_p1, _ = one_stream(0, vals_p)
    mvf = ctxs[0].mv_field()  # the plain form's last P frame: early-outs are MV 0 with SAD <= 512
    autotune.apply(vals_l)  # e2e and the full encode run the learned form
    searched = int(MBS - np.count_nonzero((mvf[:, 0] == 0) & (mvf[:, 1] == 0) & (mvf[:, 2].view(np.uint32) <= 512)))
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
    esched = GopSchedule(S)

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
            slots.append(c.encode(img, W, H, QP, esched.kind(s, k, True) == "i", 1, 0, None))
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
    ent_fps, ent_mbit = e2e_entropy(ctxs, imgs, pinned, esched, S, K, Wm, control, barrier, max_over_ranks, ws)
    for c, (img, mem) in zip(ctxs, imgs):
        c.destroy_image(img, mem)
    for c in ctxs:
        c.close()

    # ---- full encode through the reference host encoder ---------------------
    fe = {}
    if not args.no_full_encode:
        fe["learned_cavlc"] = full_encode(args, host_frames, S, K, Wm, 66, "learned_fp8")
        fe["learned_cabac"] = full_encode(args, host_frames, S, K, Wm, 77, "learned_fp8")
        fe["plain_cavlc"] = full_encode(args, host_frames, S, K, Wm, 66, "full")

    if rank == 0:
        peak, peak_kind = measured_peaks()
        pp1, pi1 = perf_l1
        nP = max(1, pp1["frames"])
        stage_ms = {k2: pp1[k2] / nP for k2 in ("me", "chain", "deblock", "staging")}
        nI = max(1, pi1["frames"])
        intra_ms = {"intra": pi1["chain"] / nI, "deblock": pi1["deblock"] / nI}
        plain_stage_ms = {k2: perf_p1[0][k2] / max(1, perf_p1[0]["frames"]) for k2 in ("me", "chain", "deblock")}
        dom = max(("me", "chain", "deblock"), key=lambda k2: stage_ms[k2])
        algo = ALGO_BYTES_PER_MB[dom] * MBS
        ach = algo / (stage_ms[dom] / 1000.0) / 1e9
        tr = traffic_from_profiles(dom)
        pipe_bytes = (ALGO_BYTES_PER_MB["me"] + ALGO_BYTES_PER_MB["chain"] + ALGO_BYTES_PER_MB["deblock"]) * MBS
        me_abs = ME_ABSDIFF_PER_MB * searched
        line = {
            "metric": METRIC, "value": round(fps, 2),
            "unit": "frames/s", "n_gpus": ws, "steps": K, "warmup": Wm,
            "ms_per_step": round(ms_l / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8/int32 (integer path), fp8 e4m3 (proposal network inference; trained in bf16)",
            "data": "synthetic (seeded generator: gradients, sigma-8 texture, 6 moving rectangles, pan, noise patch)",
            "config": bench_config(S, args.conf),
            "timed_frames": frame_kinds[LEARNED, S],
            "plain": {"value": round(fps_plain, 2), "unit": "frames/s", "ms_per_step": round(ms_p / K, 4),
                      "timed_frames": frame_kinds[0, S]},
            "speedup_vs_plain": round(fps / fps_plain, 3),
            "learned_bf16": {"value": round(fps_bf16, 2), "unit": "frames/s", "ms_per_step": round(ms_b / K, 4),
                             "speedup_vs_plain": round(fps_bf16 / fps_plain, 3),
                             "note": "the same learned form with the network's inference in BF16 (set_me mode 1)"},
            "host_issue_ms_per_step": {"learned": round(host_ms[LEARNED, S], 4), "plain": round(host_ms[0, S], 4),
                                       "note": "host time to enqueue one step (all streams); compare ms_per_step"},
            "single_stream": {"learned_fps": round(k1 / (ms_l1 / 1000.0), 2),
                              "plain_fps": round(k1 / (ms_p1 / 1000.0), 2), "frames": k1,
                              "learned_stage_ms_per_p_frame": {k2: round(v, 4) for k2, v in stage_ms.items()},
                              "plain_stage_ms_per_p_frame": {k2: round(v, 4) for k2, v in plain_stage_ms.items()},
                              "stage_ms_per_i_frame": {k2: round(v, 4) for k2, v in intra_ms.items()},
                              "last_p_frame_mbs": dict(zip(("learned", "fallback", "early"), me_counts)),
                              "deblock_tile": "8 x 8 macroblocks (the latency choice); the 8-stream arms use the "
                                              "tuned shape in `tune`"},
            "me_int": {"value": round(me_abs / (plain_stage_ms["me"] / 1000.0), 1), "unit": "abs-diff/s",
                       "searched_mbs": searched,
                       "note": f"plain full search, one stream: ({2 * RANGE + 1}^2 + 16) x 256 abs-diffs per searched "
                               "MB (zero-MV early-outs of the last P frame excluded) / ME stage time"},
            "bd_rate": rd_record(),
            "gpu_launches": launches,
            "e2e": {"value": round(ent_fps, 2), "unit": "frames/s", "h2d_bytes_per_step": S * H2D_PER_STEP,
                    "d2h_bytes_per_step": int(S * (MBS * 16 + 8) + round(ent_mbit * 1e6 / 8) * S),
                    "output": "the Annex B slice NAL units of every frame (GPU CAVLC, 4 slices)",
                    "mbit_per_frame": round(ent_mbit, 4),
                    "path": "learned form through the boundary with host buffers: pinned upload, GPU stages, GPU "
                            "CAVLC slice data into mapped host memory, slice NAL units assembled on the host (one "
                            "thread per stream)"},
            "e2e_staging": {"value": round(e2e_fps, 2), "unit": "frames/s", "h2d_bytes_per_step": S * H2D_PER_STEP,
                            "d2h_bytes_per_step": S * D2H_PER_STEP,
                            "path": "the reference boundary's staged levels, DC, nz masks, modes and vectors read "
                                    "back every step (what the reference's host entropy coder consumes)"},
            "full_encode": fe or None,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(ach / peak, 5), "peak_kind": peak_kind,
                         "traffic": (round(tr * MBS) if tr is not None else None),
                         "algorithmic_bytes": int(algo),
                         "timing": "single-stream learned run, stage events on the context stream"},
            "hbm_pipeline": {"achieved": round(pipe_bytes * fps / ws / 1e9, 2), "unit": "GB/s",
                             "frac": round(pipe_bytes * fps / ws / 1e9 / peak, 5),
                             "note": "algorithmic bytes of ME + P chain + deblock per P frame x learned-form fps"},
            "clocks": clk,
            "tune": tuned or None,
        }
        if ws == 1 and not args.no_cpu_baseline:
            spf, info = cpu_reference_frame_time(host_frames[0][:2], budget_s=15.0)
            line["cpu_baseline"] = {"value": round(1.0 / spf, 4), "unit": "frames/s", "cores": info["cores"],
                                    "kind": info["kind"], "sample": info["sample"],
                                    "stage_s": {k2: round(v, 4) for k2, v in info["stage_s"].items()}}
        print(json.dumps(line), flush=True)
    group.close()


MS_MIX = [(640, 480, 24), (1280, 720, 24), (1920, 1080, 12), (2560, 1440, 4)]
MS_RESIDENT = 8


def _ms_frames(w, h, seed, n):
    from b200enc import synth
    seq = synth.Sequence(w, h, seed=seed, pan=True, noise_patch=w >= 1280)
    return [seq.frame(t) for t in range(n)]


def run_multistream(args):
    """The batched multi-stream workload: 64 concurrent streams (24 x
    640x480, 24 x 1280x720, 12 x 1920x1080, 4 x 2560x1440), per-stream QP
    uniform in 20..40 (seeded), IPPP with an IDR every 60 frames and the
    streams' IDRs spread over the GOP, search range 32. A step is one frame
    of every stream through b200enc_batch_encode (one launch per stage for
    all 64 streams, each step a captured CUDA graph), in the plain and the
    learned (FP8 network) forms, device-timed with CUDA events on the
    batch's stream; the same streams through 64 independent single-stream
    contexts (one CUDA stream each, ~12 launches per frame) are timed beside
    them. Each stream cycles 8 resident synthetic frames (>= 800 MB in all,
    larger than L2). Prints one JSON line."""
    import multiprocessing as mp
    import numpy as np
    import torch
    import b200enc
    sizes = [(w, h) for (w, h, n) in MS_MIX for _ in range(n)]
    S = len(sizes)
    rs = np.random.Generator(np.random.PCG64(4))
    qps = [int(q) for q in rs.integers(20, 41, S)]
    phase = [(s * GOP) // S for s in range(S)]
    with mp.get_context("spawn").Pool(max(1, (os.cpu_count() or 2) - 1)) as pool:
        host = pool.starmap(_ms_frames, [(w, h, 500 + s, MS_RESIDENT) for s, (w, h) in enumerate(sizes)])
    dev = [[b200enc.NV12.from_host(y, uv) for (y, uv) in fr] for fr in host]
    mbs_per_step = sum(((w + 15) // 16) * ((h + 15) // 16) for (w, h) in sizes)

    def kinds(t):
        return [t == 0 or (t + phase[s]) % GOP == 0 for s in range(S)]

    from b200enc import autotune
    tuned = {}

    def time_batch(me_mode, graph, tune=False):
        b = b200enc.Batch(sizes, search_range=RANGE, me_mode=me_mode, deblock=1, graph=graph)
        st = torch.cuda.ExternalStream(b.stream())
        t = 0
        for _ in range(args.warmup):
            b.encode([dev[s][t % MS_RESIDENT] for s in range(S)], qps, kinds(t))
            t += 1
        assert b.sync() == 0
        if tune and not args.no_tune:
            # launch shapes for this form's batched throughput: 4 steps per
            # score, median of 3, on the same batch (steps continue the GOPs)
            tt = [t]

            def run4():
                a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a0.record(st)
                for _ in range(4):
                    b.encode([dev[s][tt[0] % MS_RESIDENT] for s in range(S)], qps, kinds(tt[0]))
                    tt[0] += 1
                a1.record(st)
                assert b.sync() == 0
                return a0.elapsed_time(a1)
            # the knobs a batch reads at every step (its P chain and full
            # search have one shape): the deblocking tile and the learned
            # form's persistent grids
            names = ["deblock_tile_w", "deblock_tile_h"] + (
                ["rescore_ctas_per_sm", "fallback_ctas_per_sm"] if me_mode else [])
            h0 = time.perf_counter()
            vals, _ = autotune.tune_throughput(run4, max(h for _, h in sizes) // 16, names, reps=3)
            tuned["learned" if me_mode else "plain"] = {"values": {n: vals[n] for n in names},
                                                        "seconds": round(time.perf_counter() - h0, 2)}
            t = tt[0]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        h0 = time.perf_counter()
        for _ in range(args.steps):
            b.encode([dev[s][t % MS_RESIDENT] for s in range(S)], qps, kinds(t))
            t += 1
        host_s = time.perf_counter() - h0
        e1.record(st)
        assert b.sync() == 0
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        gs = b.graph_stats()
        b.close()
        return ms, host_s, gs

    def time_contexts(me_mode):
        ctxs = []
        for s in range(S):
            c = b200enc.Context()
            c.configure(search_range=RANGE, lam=LAMBDA, zero_thresh=512, coded_clamp=True, deblock=1)
            c.set_me(me_mode)
            ctxs.append(c)
        streams = [torch.cuda.ExternalStream(c.stream()) for c in ctxs]
        control = torch.cuda.Stream()
        t = 0

        def step(t):
            k = kinds(t)
            for s, c in enumerate(ctxs):
                w, h = sizes[s]
                c.encode_device(dev[s][t % MS_RESIDENT], w, h, qps[s], k[s], 1, False)

        for _ in range(args.warmup):
            step(t)
            t += 1
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(control)
        for x in streams:
            x.wait_event(e0)
        for _ in range(args.steps):
            step(t)
            t += 1
        for x in streams:
            ev = torch.cuda.Event()
            ev.record(x)
            control.wait_event(ev)
        e1.record(control)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        for c in ctxs:
            c.close()
        return ms

    res = {}
    for name, mode in (("learned", LEARNED), ("plain", 0)):
        ms, host_s, gs = time_batch(mode, True, tune=mode != 0)
        res[name] = {"value": round(S * args.steps / (ms / 1000.0), 2), "unit": "frames/s",
                     "mb_per_s": round(mbs_per_step * args.steps / (ms / 1000.0), 1),
                     "ms_per_step": round(ms / args.steps, 4),
                     "host_issue_ms_per_step": round(1000.0 * host_s / args.steps, 4),
                     "graph_instantiations_updates": list(gs)}
        ms_c = time_contexts(mode)
        res[name + "_contexts"] = {"value": round(S * args.steps / (ms_c / 1000.0), 2), "unit": "frames/s",
                                   "ms_per_step": round(ms_c / args.steps, 4),
                                   "note": "the same streams through 64 single-stream contexts"}
    autotune.apply({k: 0 for k in autotune.KEYS})
    if "learned" in tuned:
        autotune.apply(tuned["learned"]["values"])
    ms_d, _, _ = time_batch(LEARNED, False)
    res["learned_no_graph"] = {"value": round(S * args.steps / (ms_d / 1000.0), 2), "unit": "frames/s",
                               "ms_per_step": round(ms_d / args.steps, 4)}
    line = {"metric": "batched multi-stream H.264 encode fps (64 streams, mixed resolutions)",
            "value": res["learned"]["value"], "unit": "frames/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["learned"]["ms_per_step"], "higher_is_better": True,
            "dtype": "u8/int32 (integer path), fp8 e4m3 (proposal network inference)",
            "data": "synthetic (seeded generator per stream)",
            "config": {"workload": "h264_multistream_64_mixed_batched", "streams": S,
                       "mix": [f"{n}x{w}x{h}" for (w, h, n) in MS_MIX], "qp": "uniform 20..40 per stream (seeded)",
                       "search_range": RANGE, "gop": GOP, "gop_phase": "stream s: s*gop/streams",
                       "deblock": True, "resident_frames_per_stream": MS_RESIDENT,
                       "l2": f"{sum(f.buf.numel() for fr in dev for f in fr) >> 20} MiB resident > L2"},
            "macroblocks_per_step": mbs_per_step, **res,
            "speedup_vs_plain": round(res["learned"]["value"] / res["plain"]["value"], 3),
            "batch_vs_contexts": round(res["learned"]["value"] / res["learned_contexts"]["value"], 3),
            "tune": tuned or None}
    print(json.dumps(line), flush=True)


def run_hevc(args):
    """HEVC encode through the reference's host encoder (hevc_encoder_encode_raw;
    wavefront rows on all host threads, QP 27 pinned, 1920x1080, 8-bit and
    Main10) as shipped (oracle/_ref/libhevcref.so) and with its half-sample
    planes built on the GPU (oracle/_ref/libhevcenc_b200.so, the binding in
    bc250-vaapi_b200/binding/hevc_hpel_binding.c): frames/s by wall clock
    over `steps` frames after `warmup` frames. The two streams are byte for
    byte the same (tests/test_gpu_hevc_encode.py). Prints one JSON line."""
    import ctypes
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import test_gpu_hevc_encode as he
    n = args.warmup + args.steps
    res = {}
    for bd in (8, 10):
        frames = he.frames_8bit(W, H, min(n, 30), 7) if bd == 8 else he.frames_p010(W, H, min(n, 30), 7)
        for name, so in (("reference", he.REF_SO), ("gpu_hpel", he.GPU_SO)):
            os.environ["BC250_HEVC_QP"] = "27"
            L = ctypes.CDLL(so)
            L.hevc_encoder_create_depth.restype = ctypes.c_void_p
            L.hevc_encoder_create_depth.argtypes = [ctypes.c_void_p] + [ctypes.c_uint32] * 4 + [ctypes.c_int]
            L.hevc_encoder_set_gop_size.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
            L.hevc_encoder_encode_raw.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
            L.hevc_encoder_destroy.argtypes = [ctypes.c_void_p]
            e = L.hevc_encoder_create_depth(None, W, H, 30, 8_000_000, bd)
            os.environ.pop("BC250_HEVC_QP", None)
            L.hevc_encoder_set_gop_size(e, GOP)
            out = np.zeros(W * H * 6, np.uint8)
            t0 = None
            nbytes = 0
            for k in range(n):
                if k == args.warmup:
                    t0 = time.perf_counter()
                y, uv = frames[k % len(frames)]
                r = L.hevc_encoder_encode_raw(e, y.ctypes.data, y.strides[0], uv.ctypes.data, uv.strides[0],
                                              out.ctypes.data, out.nbytes)
                assert r > 0
                if k >= args.warmup:
                    nbytes += r
            dt = time.perf_counter() - t0
            L.hevc_encoder_destroy(e)
            res[f"{name}_{bd}bit"] = {"value": round(args.steps / dt, 2), "unit": "frames/s",
                                      "mbit_per_frame": round(8 * nbytes / args.steps / 1e6, 4)}
    line = {"metric": "HEVC 1080p encode fps (reference host encoder, half-sample planes on the GPU)",
            "value": res["gpu_hpel_8bit"]["value"], "unit": "frames/s", "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "host_cores": os.cpu_count(),
            "config": {"workload": "hevc_1080p_wpp_qp27", "width": W, "height": H, "qp": 27, "gop": GOP,
                       "threads": os.cpu_count()}, **res,
            "note": "wall clock per frame through hevc_encoder_encode_raw; the RD loop, CABAC and the other "
                    "primitives stay on the host cores"}
    print(json.dumps(line), flush=True)


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
    ap.add_argument("--no-full-encode", action="store_true", help="skip the full-encode figure (host entropy coding)")
    ap.add_argument("--no-tune", action="store_true", help="built-in launch parameters instead of autotuned ones")
    ap.add_argument("--profile-arm", choices=["learned", "plain", "learned_bf16"], default=None,
                    help="run only this S-stream arm (warm-up + steps) and print nothing: a profiler's launch list")
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--conf", type=float, default=0.9)
    ap.add_argument("--workload", choices=["h264_1080p", "multistream", "hevc"], default="h264_1080p",
                    help="multistream: the 64-stream mixed-resolution batch (own JSON line)")
    ap.add_argument("--hevc-deblock", action="store_true",
                    help="time b200enc_hevc_deblock instead of the H.264 encode (own JSON lines)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.hevc_deblock:
        run_hevc_deblock(args)
    elif args.workload == "multistream" and args.impl != "reference":
        run_multistream(args)
    elif args.workload == "hevc" and args.impl != "reference":
        run_hevc(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
