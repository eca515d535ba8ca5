"""CPU oracle of the learned motion-proposal network. TEST INFRASTRUCTURE
ONLY: tests compare the CUDA path (csrc/proposal.cu, csrc/tc_gemm.cu)
against it; nothing in the product imports it.

The reference (MTSistemi/bc250-vaapi) has no learned part, so there is no
reference code or golden vector to pin this to. The restatement is pinned
instead by (a) central finite differences of its own FP64 forward pass
(tests/test_proposal_oracle.py) and (b) a direct image-grid convolution that
the Morton-row GEMM formulation must reproduce.

Arithmetic mirrors the CUDA path's cast points: GEMM operands are BF16
(round to nearest even), accumulation FP32 (emulated here in FP64, then
rounded to FP32), bias and ReLU in FP32, hidden outputs rounded to BF16,
logits FP32; the loss gradient is rounded to BF16 before the backward GEMMs,
ReLU masks come from the BF16 outputs, and each layer's input gradient is
FP32 before masking and rounding. With `exact=True` every rounding is off
(FP64 throughout), which is what the finite-difference check uses.
"""
import numpy as np

LAYERS = [(8, 32), (128, 32), (128, 32), (128, 32), (96, 64), (64, 16)]
N_CAND, N_CLASSES, N_OUT = 10, 11, 16


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even); returns float32."""
    x = np.ascontiguousarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(params):
    out, o = [], 0
    for i, n in LAYERS:
        W = params[o:o + n * i].reshape(n, i)
        b = params[o + n * i:o + n * i + n]
        out.append((W, b))
        o += n * i + n
    return out


def _gemm(A, W, exact):
    """A [rows][in] . W[out][in]^T with BF16 operands and FP32 accumulation."""
    if exact:
        return A.astype(np.float64) @ W.astype(np.float64).T
    return (bf16(A).astype(np.float64) @ bf16(W).astype(np.float64).T).astype(np.float32)


def forward(params, x0, side, exact=False):
    """x0: [B*64][8] network input rows (Morton order per MB); side: [B][64]
    side features. Returns (logits [B][16], activations)."""
    L = unpack(params.astype(np.float64) if exact else params)
    B = side.shape[0]
    rnd = (lambda v: v) if exact else bf16
    acts = {"a0": x0}
    a = x0
    for l in range(4):
        W, b = L[l]
        z = _gemm(a, W, exact) + b
        y = rnd(np.maximum(z, 0))
        acts[f"y{l}"] = y
        a = y.reshape(-1, 128) if l < 3 else y
    f = np.concatenate([acts["y3"], side], axis=1)
    acts["f"] = f
    W, b = L[4]
    h = rnd(np.maximum(_gemm(f, W, exact) + b, 0))
    acts["h"] = h
    W, b = L[5]
    logits = _gemm(h, W, exact) + b
    if not exact:
        logits = logits.astype(np.float32)
    assert logits.shape == (B, N_OUT)
    return logits, acts


FP8_MAX = np.float32(448.0)
NET8_TILE = 16


def e4m3(x):
    """Round float32 values to FP8 E4M3 (the 'fn' variant: largest finite
    448, no infinities), nearest with ties to even, saturating at +-448;
    returns float32. torch's float8_e4m3fn conversion does the rounding."""
    import torch
    t = torch.from_numpy(np.clip(np.ascontiguousarray(x, np.float32), -FP8_MAX, FP8_MAX))
    return t.to(torch.float8_e4m3fn).to(torch.float32).numpy()


def _e4m3_scale(amax):
    """(multiplier that quantises, multiplier that undoes it) of a maximum."""
    amax = np.float32(amax)
    if amax > 0:
        return np.float32(FP8_MAX / amax), np.float32(amax / FP8_MAX)
    return np.float32(1.0), np.float32(1.0)


def quantize_weights_fp8(params):
    """Per-output-channel E4M3 weights of every layer: [(W8, s_w, b)], W8
    holding the E4M3 values as float32 (csrc/proposal_infer8.cu stage_w8)."""
    out = []
    for W, b in unpack(np.asarray(params, np.float32)):
        W = W.astype(np.float32)
        amax = np.abs(W).max(axis=1).astype(np.float32)
        safe = np.where(amax > 0, amax, np.float32(1)).astype(np.float32)
        inv = np.where(amax > 0, FP8_MAX / safe, np.float32(1)).astype(np.float32)
        sw = np.where(amax > 0, safe / FP8_MAX, np.float32(1)).astype(np.float32)
        out.append((e4m3(W * inv[:, None]), sw, b.astype(np.float32)))
    return out


def _fma32(acc, sc, b):
    """float32(acc * sc + b) with one rounding (fmaf), via float64."""
    return (acc.astype(np.float64) * sc.astype(np.float64) + b.astype(np.float64)).astype(np.float32)


def forward_fp8(params, x0, side):
    """The FP8 inference form (csrc/proposal_infer8.cu): per 16-MB tile, the
    network input, each hidden output after bias and ReLU, and the fc1 input
    (c4 output with the side features) are quantised to E4M3 with one scale
    per tile (amax / 448); weights with one scale per output channel; E4M3
    products accumulate in FP32 (here FP64, then rounded); each epilogue is
    fma(acc, s_in * s_w, b). A last partial tile is padded with zero MBs, as
    the kernel does. Returns logits [B][16] (float32)."""
    Q = quantize_weights_fp8(params)
    B = side.shape[0]
    T = NET8_TILE
    logits = np.zeros((B, N_OUT), np.float32)
    for t0 in range(0, B, T):
        n = min(T, B - t0)
        x = np.zeros((T * 64, 8), np.float32)
        x[:n * 64] = x0[t0 * 64:(t0 + n) * 64]
        sd = np.zeros((T, 64), np.float32)
        sd[:n] = side[t0:t0 + n]
        inv, s = _e4m3_scale(np.abs(x).max())
        a8 = e4m3(x * inv)
        for l in range(5):
            W8, sw, b = Q[l]
            acc = (a8.astype(np.float64) @ W8.astype(np.float64).T).astype(np.float32)
            y = np.maximum(_fma32(acc, (s * sw).astype(np.float32), b), np.float32(0))
            if l < 3:
                y = y.reshape(-1, 128)
            elif l == 3:
                y = np.concatenate([y, sd], axis=1)
            inv, s = _e4m3_scale(np.abs(y).max())
            a8 = e4m3(y * inv)
        W8, sw, b = Q[5]
        acc = (a8.astype(np.float64) @ W8.astype(np.float64).T).astype(np.float32)
        logits[t0:t0 + n] = _fma32(acc, (s * sw).astype(np.float32), b)[:n]
    return logits


def _masked_softmax(z, dup):
    valid = np.ones_like(z[:, :N_CLASSES], bool)
    valid[:, :N_CAND] = ((dup[:, None] >> np.arange(N_CAND)[None, :]) & 1) == 0
    zz = np.where(valid, z[:, :N_CLASSES], -np.inf)
    m = zz.max(axis=1, keepdims=True)
    e = np.where(valid, np.exp(zz - m), 0.0)
    return e / e.sum(axis=1, keepdims=True)


def loss_and_grad(logits, label, norez, weight, dup):
    """Mean over weighted samples of -log(probability mass of the target set
    `label` (bit mask over the 11 classes) under the masked softmax) + 0.5 BCE
    on logit 11. Returns (loss, dloss/dlogits [B][16])."""
    z = logits.astype(np.float64)
    p = _masked_softmax(z, dup)
    n = max(float((weight > 0).sum()), 1.0)
    w = weight.astype(np.float64) / n
    B = z.shape[0]
    inset = ((np.asarray(label, np.int64)[:, None] >> np.arange(N_CLASSES)[None, :]) & 1).astype(bool)
    pset = np.maximum((p * inset).sum(axis=1), 1e-30)
    g = np.zeros((B, N_OUT))
    g[:, :N_CLASSES] = w[:, None] * (p - np.where(inset, p / pset[:, None], 0.0))
    zs = z[:, 11]
    ps = 1.0 / (1.0 + np.exp(-zs))
    g[:, 11] = w * 0.5 * (ps - norez)
    ce = -np.log(pset)
    bce = np.maximum(zs, 0) - zs * norez + np.log1p(np.exp(-np.abs(zs)))
    loss = float(np.sum(np.where(weight > 0, w * (ce + 0.5 * bce), 0.0)))
    return loss, g


def backward(params, acts, g5, exact=False):
    """Gradients (flat, like params) of the loss whose logit gradient is g5."""
    L = unpack(params.astype(np.float64) if exact else params)
    rnd = (lambda v: v) if exact else bf16
    grads = []

    def layer(l, G, A):
        W, _ = L[l]
        Gd = G.astype(np.float64)
        gW = Gd.T @ A.astype(np.float64)
        gb = Gd.sum(axis=0)
        dA = Gd @ (W.astype(np.float64) if exact else bf16(W).astype(np.float64))
        if not exact:
            gW, gb, dA = gW.astype(np.float32), gb.astype(np.float32), dA.astype(np.float32)
        grads.append((l, gW, gb))
        return dA

    G = rnd(g5.astype(np.float32) if not exact else g5)
    dA = layer(5, G, acts["h"])
    G = rnd(dA * (acts["h"] > 0))
    dA = layer(4, G, acts["f"])
    G = rnd(dA[:, :32] * (acts["y3"] > 0))
    dA = layer(3, G, acts["y2"].reshape(-1, 128))
    G = rnd(dA.reshape(-1, 32) * (acts["y2"] > 0))
    dA = layer(2, G, acts["y1"].reshape(-1, 128))
    G = rnd(dA.reshape(-1, 32) * (acts["y1"] > 0))
    dA = layer(1, G, acts["y0"].reshape(-1, 128))
    G = rnd(dA.reshape(-1, 32) * (acts["y0"] > 0))
    layer(0, G, acts["a0"])
    flat = np.zeros(sum(n * i + n for i, n in LAYERS), np.float64)
    offs, o = [], 0
    for i, n in LAYERS:
        offs.append(o)
        o += n * i + n
    for l, gW, gb in grads:
        i, n = LAYERS[l]
        flat[offs[l]:offs[l] + n * i] = gW.reshape(-1)
        flat[offs[l] + n * i:offs[l] + n * i + n] = gb
    return flat


# ---------------------------------------------------------------- preparation
NB = [(0, 0), (-1, -1), (0, -1), (1, -1), (-1, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]


def morton_xy(m):
    x = (m & 1) | ((m >> 1) & 2) | ((m >> 2) & 4)
    y = ((m >> 1) & 1) | ((m >> 2) & 2) | ((m >> 3) & 4)
    return x, y


def _f32(v):
    return np.float32(v)


def prepare(cur, ref, W, H, RW, RH, prev_mv, R, zero_thresh):
    """Candidates, exact SADs, state words, network input and side features of
    every MB, as lp_prepare_kernel computes them. cur [>=H][>=W], ref
    [>=RH][>=RW] uint8; prev_mv [mbs][4] int32 (mvx, mvy, sad, pad) or None."""
    mbw, mbh = (W + 15) // 16, (H + 15) // 16
    mbs = mbw * mbh
    cand = np.zeros((mbs, N_CAND, 2), np.int32)
    csad = np.zeros((mbs, N_CAND), np.uint32)
    state = np.zeros(mbs, np.uint32)
    x0 = np.zeros((mbs * 64, 8), np.float32)
    side = np.zeros((mbs, 64), np.float32)
    ys = np.arange(16)
    for mb in range(mbs):
        mby, mbx = divmod(mb, mbw)
        X, Y = mbx * 16, mby * 16
        c = cur[np.clip(Y + ys, 0, H - 1)][:, np.clip(X + ys, 0, W - 1)].astype(np.int64)
        sprev = np.zeros(9, np.int64)
        for k in range(N_CAND):
            cx = cy = 0
            if k < 9 and prev_mv is not None:
                nx = min(max(mbx + NB[k][0], 0), mbw - 1)
                ny = min(max(mby + NB[k][1], 0), mbh - 1)
                m = prev_mv[ny * mbw + nx]
                cx = min(max((int(m[0]) + 2) >> 2, -(R - 2)), R - 2)
                cy = min(max((int(m[1]) + 2) >> 2, -(R - 2)), R - 2)
                sprev[k] = int(np.uint32(m[2]))
            cand[mb, k] = (cx, cy)
            r = ref[np.clip(Y + ys + cy, 0, RH - 1)][:, np.clip(X + ys + cx, 0, RW - 1)].astype(np.int64)
            csad[mb, k] = np.abs(c - r).sum()
        dup = 0
        for k in range(N_CAND):
            for d in range(k):
                if tuple(cand[mb, d]) == tuple(cand[mb, k]):
                    dup |= 1 << k
                    break
        early = zero_thresh >= 0 and int(csad[mb, 9]) <= zero_thresh
        state[mb] = (1 if early else 0) | (0 if prev_mv is not None else 2) | (dup << 8)
        c0x, c0y = cand[mb, 0]
        r0 = ref[np.clip(Y + ys + c0y, 0, RH - 1)][:, np.clip(X + ys + c0x, 0, RW - 1)].astype(np.int64)
        for m in range(64):
            ox, oy = morton_xy(m)
            for dy in range(2):
                for dx in range(2):
                    y, x = 2 * oy + dy, 2 * ox + dx
                    x0[mb * 64 + m, (dy * 2 + dx) * 2] = _f32(c[y, x] - 128) * _f32(0.015625)
                    x0[mb * 64 + m, (dy * 2 + dx) * 2 + 1] = _f32(c[y, x] - r0[y, x]) * _f32(0.015625)
        smin = int(csad[mb].min())
        s = csad[mb].astype(np.int64)
        f = np.zeros(64, np.float32)
        f[0:10] = np.minimum(s, 32767).astype(np.float32) * _f32(1 / 4096)
        f[10:20] = np.minimum(s - smin, 32767).astype(np.float32) * _f32(1 / 4096)
        f[20:30] = (cand[mb, :, 0] - c0x).astype(np.float32) * _f32(0.125)
        f[30:40] = (cand[mb, :, 1] - c0y).astype(np.float32) * _f32(0.125)
        f[40:50] = [(dup >> k) & 1 for k in range(N_CAND)]
        f[50:59] = np.minimum(sprev, 32767).astype(np.float32) * _f32(1 / 4096)
        f[59] = _f32(abs(c0x)) * _f32(0.03125)
        f[60] = _f32(abs(c0y)) * _f32(0.03125)
        f[61] = _f32(np.abs(np.diff(c, axis=1)).sum()) / _f32(7680)
        f[62] = _f32(np.abs(np.diff(c, axis=0)).sum()) / _f32(7680)
        f[63] = 0.0 if prev_mv is not None else 1.0
        side[mb] = f
    return dict(cand=cand, cand_sad=csad, state=state, x0=bf16(x0), side=bf16(side))


def labels(state, cand, logged_pad, nz=None):
    """Training targets from full-search log words (see lp_label_kernel):
    a bit mask of the distinct candidates whose +-2 window holds the integer
    winner, or of class 10 ("none") when no window does."""
    mbs = state.shape[0]
    lab = np.zeros(mbs, np.int32)
    w = np.zeros(mbs, np.float32)
    pad = logged_pad.astype(np.uint32)
    for mb in range(mbs):
        valid = (pad[mb] >> 31) and not ((pad[mb] >> 30) & 1) and not (state[mb] & 3)
        if not valid:
            continue
        w[mb] = 1
        dx, dy = int(pad[mb] & 0xFF) - 128, int((pad[mb] >> 8) & 0xFF) - 128
        dup = int(state[mb] >> 8) & 0x3FF
        for k in range(N_CAND):
            if (dup >> k) & 1:
                continue
            if abs(dx - cand[mb, k, 0]) <= 2 and abs(dy - cand[mb, k, 1]) <= 2:
                lab[mb] |= 1 << k
    lab[lab == 0] = 1 << (N_CLASSES - 1)
    norez = np.ones(mbs, np.float32) if nz is None else (nz.reshape(mbs, -1) == 0).all(axis=1).astype(np.float32)
    return lab, norez, w


def select(logits, state, conf):
    """(sel [mbs][4] candidate indices or -1, is_learned, is_fallback)."""
    mbs = logits.shape[0]
    sel = np.full((mbs, 4), -1, np.int32)
    learned = np.zeros(mbs, bool)
    fallback = np.zeros(mbs, bool)
    dup = (state >> 8) & 0x3FF
    p = _masked_softmax(logits.astype(np.float64), dup.astype(np.int64))
    for mb in range(mbs):
        if state[mb] & 1:
            continue
        if state[mb] & 2:
            fallback[mb] = True
            continue
        chosen = int(dup[mb])
        c_sum = 0.0
        for k in range(4):
            best = -1
            for c in range(N_CAND):
                if not (chosen >> c) & 1 and (best < 0 or p[mb, c] > p[mb, best]):
                    best = c
            if best < 0:
                break
            chosen |= 1 << best
            c_sum += p[mb, best]
            sel[mb, k] = best
        (fallback if c_sum < conf else learned)[mb] = True
    return sel, learned, fallback
