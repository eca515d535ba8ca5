"""Trains the learned motion-proposal network on decisions logged by the plain
full-search encoder, on the GPU, with the library's own kernels.

Data: seeded synthetic sequences (b200enc.synth, the 1080p workload's
content model: gradients, static texture, six moving rectangles, global pan,
a uniform-noise patch), each encoded by the plain stages (I frame, then P
frames: full search -> transform/quant/recon -> deblock) at a QP of
22/27/32/37 in turn. Every P frame from the third on is a training sample:
the current frame, the deblocked reference, the previous frame's MV field
(the candidates) and the full search's integer winners (the targets, logged
with B200ENC_ME_LOG_INTEGER) and nz words (the no-residual target).
Held-out sequences (other seeds) give the validation figures written into
the checkpoint's metadata.

    python -m b200enc.train_proposal --out weights.b2pn [--sequences 200]
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import time

import numpy as np

QPS = (22, 27, 32, 37)


def _gen_sequence(args):
    """Frames of one synthetic sequence (runs in a worker process)."""
    W, H, seed, frames = args
    from b200enc import synth
    seq = synth.Sequence(W, H, seed=seed, pan=True, noise_patch=True)
    return [seq.frame(t) for t in range(frames)]


def generate(W, H, seeds, frames, workers=None):
    """Frames of every sequence, generated on the host cores. The pool is
    started with 'spawn' so that no CUDA state is forked."""
    ctx = mp.get_context("spawn")
    workers = workers or max(1, min(len(seeds), (os.cpu_count() or 2) - 1, 32))
    with ctx.Pool(workers) as pool:
        return pool.map(_gen_sequence, [(W, H, s, frames) for s in seeds], chunksize=1)


class Sample:
    __slots__ = ("cur", "ref", "prev", "logged", "nz", "qp")

    def __init__(self, cur, ref, prev, logged, nz, qp):
        self.cur, self.ref, self.prev, self.logged, self.nz, self.qp = cur, ref, prev, logged, nz, qp


def encode_log(frames, W, H, qp, R=32, lam=5, zero_thresh=512):
    """Plain-form encode of one sequence with the stage kernels; returns the
    training samples of its P frames from the third frame on."""
    import torch
    import b200enc as gpu
    CW, CH = gpu.coded(W, H)
    mbw, mbh = CW // 16, CH // 16
    mbs = mbw * mbh
    scr = gpu.scratch(mbh)
    nv = [gpu.NV12.from_host(y, uv) for y, uv in frames]
    out = gpu.Outputs(W, H)
    rec = gpu.NV12(W, H)
    gpu.i_frame(nv[0], W, H, CW, CH, qp, 1, out, rec, scr)
    gpu.deblock(mbw, mbh, qp, 1, out.nz, out.mv, rec, scr)
    prev_mv = None
    samples = []
    for t in range(1, len(frames)):
        mv = torch.zeros((mbs, 4), dtype=torch.int32, device="cuda")
        gpu.me_full_search_ex(nv[t], rec, W, H, CW, CH, R, lam, zero_thresh, mv, flags=gpu.ME_LOG_INTEGER)
        o = gpu.Outputs(W, H)
        new_rec = gpu.NV12(W, H)
        gpu.p_frame(nv[t], rec, W, H, CW, CH, qp, mv, o, new_rec)
        gpu.deblock(mbw, mbh, qp, 0, o.nz, mv, new_rec, scr)
        if prev_mv is not None:
            samples.append(Sample(nv[t], rec, prev_mv, mv, o.nz, qp))
        prev_mv = mv
        rec = new_rec
    return samples


def lr_at(step, total, lr_max, warmup=50, lr_min_frac=0.05):
    if step <= warmup:
        return lr_max * step / warmup
    t = (step - warmup) / max(1, total - warmup)
    return lr_max * (lr_min_frac + (1 - lr_min_frac) * 0.5 * (1 + math.cos(math.pi * min(t, 1.0))))


NET_CONF = (0.5, 0.7, 0.8, 0.9, 0.95, 0.98)
CAND_COST = (-1.0, 24.0, 16.0, 12.0, 8.0, 6.0, 4.0, 3.0)  # fallback cost per pel of the no-network baseline


def evaluate(P, samples, W, H, R=32, lam=5, net_conf=NET_CONF, cand_cost=CAND_COST, net_mode=None):
    """Validation figures over held-out samples, for the network at each
    confidence threshold and for the same candidate search without the
    network at each fallback cost threshold. A 'miss' is an MB that did not
    fall back and whose full-search integer winner lies outside the selected
    candidates' +-2 windows, i.e. whose MV may differ from the plain
    search's; rates are over MBs that are neither zero-MV early-outs nor
    without history. 'gain' compares, at the network's fallback rate, the
    baseline's miss rate (interpolated along its threshold sweep) with the
    network's. net_mode: the ME mode of the network (BF16 by default)."""
    import torch
    import b200enc as gpu
    from b200enc import proposal as pp
    CW, CH = gpu.coded(W, H)
    mbs = (CW // 16) * (CH // 16)
    net_mode = pp.Proposal.NETWORK if net_mode is None else net_mode
    configs = [("net", net_mode, c) for c in net_conf] + \
              [("cand", pp.Proposal.CANDIDATES, c) for c in cand_cost]
    stats = {(k, c): dict(valid=0, fallback=0, miss=0) for k, _, c in configs}
    top1 = 0
    nval = 0
    out = torch.zeros((mbs, 4), dtype=torch.int32, device="cuda")
    ar = np.arange(mbs)
    for s in samples:
        pad = s.logged.cpu().numpy()[:, 3].astype(np.uint32)
        wx = (pad & 0xFF).astype(np.int64) - 128
        wy = ((pad >> 8) & 0xFF).astype(np.int64) - 128
        for kind, mode, c in configs:
            P.me(s.cur, s.ref, W, H, CW, CH, s.prev, R, lam, 512, c, out, mode=mode)
            torch.cuda.synchronize()
            state = P.tensor(pp.T_STATE, torch.int32, (mbs,)).cpu().numpy().view(np.uint32)
            sel = P.tensor(pp.T_SEL, torch.int32, (mbs,)).cpu().numpy().view(np.uint32)
            cnt = P.counters()
            lists = P.tensor(pp.T_LISTS, torch.int32, (2 * mbs,)).cpu().numpy()
            fb = np.zeros(mbs, bool)
            fb[lists[mbs:mbs + cnt[1]]] = True
            cand = P.tensor(pp.T_CAND, torch.int32, (mbs, 10)).cpu().numpy().astype(np.int64)
            cx = ((cand & 0xFFFF) ^ 0x8000) - 0x8000
            cy = cand >> 16
            valid = ((pad >> 31) == 1) & (((pad >> 30) & 1) == 0) & ((state & 3) == 0)
            covered = np.zeros(mbs, bool)
            for k in range(4):
                ck = ((sel >> (8 * k)) & 0xFF).astype(np.int64)
                ok = ck < 10
                ci = np.where(ok, ck, 0)
                covered |= ok & (np.abs(wx - cx[ar, ci]) <= 2) & (np.abs(wy - cy[ar, ci]) <= 2)
            st = stats[(kind, c)]
            st["valid"] += int(valid.sum())
            st["fallback"] += int((valid & fb).sum())
            st["miss"] += int((valid & ~fb & ~covered).sum())
            if kind == "net" and c == net_conf[0]:
                P.labels(mbs, s.logged, s.nz)
                torch.cuda.synchronize()
                lab = P.tensor(pp.T_LABEL, torch.int32, (mbs,)).cpu().numpy()
                first = (sel & 0xFF).astype(np.int64)
                top1 += int((valid & (first < 10) & (((lab >> np.minimum(first, 10)) & 1) == 1)).sum())
                nval += int(valid.sum())
    rate = {k: (st["fallback"] / max(st["valid"], 1), st["miss"] / max(st["valid"], 1)) for k, st in stats.items()}
    cand_curve = sorted(rate[("cand", c)] for c in cand_cost)  # by fallback rate
    fx = np.array([f for f, _ in cand_curve])
    my = np.array([m for _, m in cand_curve])
    res = {"top1_covering": top1 / max(nval, 1), "mbs_per_config": int(stats[configs[0][0::2]]["valid"]),
           "network": {}, "no_network": {}}
    for c in net_conf:
        f, m = rate[("net", c)]
        base = float(np.interp(f, fx, my))
        res["network"][str(c)] = {"fallback_rate": f, "miss_rate": m, "no_network_miss_at_same_fallback": base}
    for c in cand_cost:
        f, m = rate[("cand", c)]
        res["no_network"][str(c)] = {"fallback_rate": f, "miss_rate": m}
    return res


def train(out, sequences=200, val_sequences=16, frames=5, W=1920, H=1080, epochs=4, lr=2e-3, seed=0,
          report=None, log=print):
    import torch
    import b200enc as gpu
    from b200enc import proposal as pp
    t0 = time.time()
    CW, CH = gpu.coded(W, H)
    mbs = (CW // 16) * (CH // 16)
    train_seeds = [seed * 100000 + i for i in range(sequences)]
    val_seeds = [seed * 100000 + 1000000 + i for i in range(val_sequences)]
    samples, val = [], []
    chunk = 32
    for lo in range(0, len(train_seeds) + len(val_seeds), chunk):
        seeds = (train_seeds + val_seeds)[lo:lo + chunk]
        for s, fr in zip(seeds, generate(W, H, seeds, frames)):
            dst = val if s in val_seeds else samples
            dst.extend(encode_log(fr, W, H, QPS[s % len(QPS)]))
    torch.cuda.synchronize()
    log(f"logged {len(samples)} training / {len(val)} validation frames in {time.time() - t0:.1f}s")
    P = pp.Proposal(mbs, pp.init_params(seed))
    loss_t = P.tensor(pp.T_LOSS, torch.float32, (1,))
    rs = np.random.Generator(np.random.PCG64(seed))
    total = epochs * len(samples)
    step = 0
    history = []
    t1 = time.time()
    for ep in range(epochs):
        loss_t.zero_()
        for i in rs.permutation(len(samples)):
            s = samples[i]
            step += 1
            P.prepare(s.cur, s.ref, W, H, CW, CH, s.prev, 32, 512)
            P.labels(mbs, s.logged, s.nz)
            P.train_step(mbs, lr_at(step, total, lr), step)
        torch.cuda.synchronize()
        history.append(float(loss_t.cpu()[0]) / len(samples))
        log(f"epoch {ep}: mean loss {history[-1]:.4f} ({time.time() - t1:.1f}s)")
    train_s = time.time() - t1
    params = P.get_params()
    metrics = evaluate(P, val, W, H)
    log(json.dumps(metrics, indent=1))
    meta = dict(workload=f"{W}x{H} synthetic (pan, noise patch), QP {list(QPS)}, R32 lambda5", sequences=sequences,
                frames_per_sequence=frames, training_frames=len(samples), validation_frames=len(val), epochs=epochs,
                lr=lr, seed=seed, loss_history=history, train_seconds=train_s, validation=metrics)
    digest = pp.save_checkpoint(out, params, step=step, meta=meta)
    if report:
        with open(report, "w") as f:
            json.dump(dict(meta, sha256=digest), f, indent=1)
    return params, meta


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--report")
    ap.add_argument("--sequences", type=int, default=200)
    ap.add_argument("--val-sequences", type=int, default=16)
    ap.add_argument("--frames", type=int, default=5)
    ap.add_argument("--size", default="1920x1080")
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    W, H = (int(v) for v in a.size.split("x"))
    train(a.out, a.sequences, a.val_sequences, a.frames, W, H, a.epochs, a.lr, a.seed, a.report)


if __name__ == "__main__":
    main()
