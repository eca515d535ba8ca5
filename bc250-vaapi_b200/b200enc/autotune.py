"""Autotuner of the encoder's launch shapes.

The library reads eight launch parameters from a process-wide table
(include/b200enc.h, B200ENC_TUNE_*): macroblock rows per CTA of the
deblocking wavefront (the stage-level b200enc_deblock), macroblocks per
P-chain CTA (the CTA tile shape), the persistent grids of the learned form's
re-scoring and fallback search, the intra wavefront's CTA count, whether the
full search stages its reference windows by TMA or by word loads, and the
tile shape of the tile deblocking that encoding contexts and batches run.
None changes a result; each
changes how the work maps onto the 148 SMs. This module times the candidates of each on
the device for one frame size, by coordinate descent over the knobs with the
library's own per-stage CUDA-event timing (b200enc_ctx_perf), keeps the
fastest, and caches the choice per device and frame size in a JSON file; a
C caller loads the same choice from the "name value" file that
write_tune_file writes (B200ENC_TUNE_FILE). The reference has nothing to
tune: its shader dispatch sizes are fixed (gpu_compute.c).
"""
import json
import os
import time

KEYS = {"deblock_rows": 0, "pchain_mbs_per_cta": 1, "rescore_ctas_per_sm": 2, "fallback_ctas_per_sm": 3,
        "intra_ctas": 4, "me_stage": 5, "deblock_tile_w": 6, "deblock_tile_h": 7}
# the knobs an encoding context (and a batch) reads; deblock_rows shapes only
# the stage-level wavefront deblocking (b200enc_deblock)
TUNED = [n for n in KEYS if n != "deblock_rows"]
# the stage whose time each knob changes (b200enc_ctx_perf_read keys), and on which frames
STAGE = {"deblock_rows": ("deblock", False), "pchain_mbs_per_cta": ("chain", False),
         "rescore_ctas_per_sm": ("me", False), "fallback_ctas_per_sm": ("me", False),
         "intra_ctas": ("chain", True), "me_stage": ("me", False),
         "deblock_tile_w": ("deblock", False), "deblock_tile_h": ("deblock", False)}


def candidates(name, mbh):
    if name == "deblock_rows":
        return [2, 3, 4, 5, 6]
    if name == "pchain_mbs_per_cta":
        return [1, 2, 4]
    if name in ("rescore_ctas_per_sm", "fallback_ctas_per_sm"):
        return [2, 4, 8, 12, 16]
    if name == "intra_ctas":
        return sorted({max(1, mbh // 2), mbh})
    if name == "me_stage":
        return [2, 1]
    if name == "deblock_tile_w":
        return [4, 6, 8]
    if name == "deblock_tile_h":
        return [2, 4, 6, 8]
    raise KeyError(name)


def throughput_candidates(name, mbh):
    """Candidates of a knob when the objective is a many-stream workload's
    throughput: wider deblocking groups than the single-stream latency
    optimum can pay there (fewer CTAs and group boundaries per frame)."""
    if name == "deblock_rows":
        return [3, 4, 5, 6]
    if name in ("rescore_ctas_per_sm", "fallback_ctas_per_sm"):
        return [4, 8, 12, 16]
    if name == "deblock_tile_w":  # wider tiles: less margin work per frame, longer chains
        return [6, 8, 12, 16]
    return candidates(name, mbh)


def tune_throughput(run, mbh, names=None, reps=3, log=None):
    """Coordinate descent over the knobs (`names`, default all) for the
    throughput of the caller's workload: `run()` encodes a fixed number of
    steps of it and returns their device milliseconds. Each candidate is
    scored by the median of `reps` runs; the fastest value of a knob is kept
    before the next knob is tried. Returns ({name: value}, {name: {value:
    ms}}) and leaves the table set to the choice. The number of run() calls
    depends only on the candidate lists, so ranks of a multi-GPU job that
    tune side by side make the same calls (run() may hold a barrier)."""
    names = list(names or TUNED)
    best = {name: 0 for name in KEYS}
    apply(best)
    scores_all = {}
    for name in names:
        scores = {}
        for v in throughput_candidates(name, mbh):
            apply({name: v})
            t = sorted(run() for _ in range(reps))
            scores[v] = t[len(t) // 2]
        pick = min(scores, key=lambda v: (scores[v], v))
        best[name] = pick
        apply({name: pick})
        scores_all[name] = scores
        if log:
            log(f"autotune {name}: " + ", ".join(f"{v}={ms:.3f}ms" for v, ms in scores.items()) + f" -> {pick}")
    return best, scores_all


def default_cache():
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "b200enc", "tune.json")


def device_key(W, H):
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|sm{p.multi_processor_count}|{W}x{H}"


def apply(values):
    """Sets the library's table from {name: value} (unknown names ignored)."""
    from . import lib
    L = lib()
    for name, v in values.items():
        if name in KEYS and L.b200enc_tune_set(KEYS[name], int(v)) != 0:
            raise ValueError(f"tune value out of range: {name}={v}")


def current():
    from . import lib
    L = lib()
    return {name: L.b200enc_tune_get(k) for name, k in KEYS.items()}


def write_tune_file(path, values):
    """The "name value" file the library loads (B200ENC_TUNE_FILE)."""
    with open(path, "w") as f:
        f.write("# b200enc launch parameters (b200enc.autotune)\n")
        for name, v in values.items():
            f.write(f"{name} {int(v)}\n")


def _time_stage(ctx, frames, W, H, qp, stage, intra, mode, reps):
    """Median per-frame milliseconds of `stage` over `reps` passes of the
    sequence (I frame, then P frames) on one context."""
    res = []
    for _ in range(reps):
        ctx.perf(True)
        for t, fr in enumerate(frames):
            ctx.encode_device(fr, W, H, qp, t == 0, 1, False)
        d = ctx.perf_read(intra)
        ctx.perf(False)
        if d["frames"]:
            res.append(d[stage] / d["frames"])
    res.sort()
    return res[len(res) // 2] if res else float("inf")


def tune(frames, W, H, qp=27, search_range=32, lam=5, learned_mode=3, conf=0.9, reps=3, log=None):
    """Coordinate descent over the knobs on `frames` (device NV12 frames of
    one stream: frame 0 is coded intra, the rest P). Returns
    {name: value} and leaves the table set to it."""
    from . import Context
    mbh = (H + 15) // 16
    ctx = Context()
    ctx.configure(search_range=search_range, lam=lam, zero_thresh=512, coded_clamp=True, deblock=1)
    best = {name: 0 for name in KEYS}
    apply(best)
    try:
        for name in TUNED:
            stage, intra = STAGE[name]
            mode = learned_mode if name in ("rescore_ctas_per_sm", "fallback_ctas_per_sm") else 0
            ctx.set_me(mode, conf=conf)
            _time_stage(ctx, frames, W, H, qp, stage, intra, mode, 1)  # warm-up
            scores = {}
            for v in candidates(name, mbh):
                apply({name: v})
                scores[v] = _time_stage(ctx, frames, W, H, qp, stage, intra, mode, reps)
            pick = min(scores, key=lambda v: (scores[v], v))
            best[name] = pick
            apply({name: pick})
            if log:
                log(f"autotune {name}: " + ", ".join(f"{v}={ms * 1000:.1f}us" for v, ms in scores.items())
                    + f" -> {pick}")
    finally:
        ctx.close()
    return best


def load_or_tune(frames, W, H, cache=None, **kw):
    """The cached choice for this device and frame size if there is one,
    else a fresh tune (saved). Returns (values, source, seconds)."""
    path = cache or default_cache()
    key = device_key(W, H)
    db = {}
    if os.path.exists(path):
        try:
            with open(path) as f:
                db = json.load(f)
        except (OSError, ValueError):
            db = {}
    if key in db:
        apply(db[key])
        return db[key], "cache", 0.0
    t0 = time.perf_counter()
    vals = tune(frames, W, H, **kw)
    dt = time.perf_counter() - t0
    db[key] = vals
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
    except OSError:
        pass
    return vals, "tuned", dt
