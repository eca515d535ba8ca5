"""Multi-stream batches (b200enc_batch_*): streams of uneven frame sizes and
per-stream QPs through one launch per stage must give, stream by stream,
exactly what a single-stream context computes from the same frames: levels,
DC, nonzero masks, prediction modes, motion vectors and the deblocked
reconstruction, step after step, with I frames at different steps in
different streams; for the plain full search and the learned form (FP8
network), launched directly and as a captured CUDA graph per step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(640, 480), (352, 288), (1280, 720), (176, 144), (1920, 1080), (720, 576)]
QPS = [26, 33, 22, 40, 28, 35]
STEPS = 6


def _intra(s, t):
    # every stream starts intra; stream s refreshes at step 2 + s % 3 (some never within STEPS)
    return t == 0 or t == 2 + s % 4


def _frames(gpu):
    from b200enc import synth
    out = []
    for s, (w, h) in enumerate(SIZES):
        seq = synth.Sequence(w, h, seed=100 + s, pan=True, noise_patch=w >= 1280)
        out.append([gpu.NV12.from_host(*seq.frame(t)) for t in range(STEPS)])
    return out


def _single(gpu, frames, me_mode):
    """Per stream, per step: the single-stream context's outputs."""
    res = []
    for s, (w, h) in enumerate(SIZES):
        ctx = gpu.Context()
        ctx.configure(search_range=32, lam=5, zero_thresh=512, coded_clamp=True, deblock=1)
        ctx.set_me(me_mode)
        per = []
        for t in range(STEPS):
            ctx.encode_device(frames[s][t], w, h, QPS[s], _intra(s, t), 1, False)
            y, uv = ctx.recon_host()
            import ctypes
            ptrs = [ctypes.c_void_p() for _ in range(5)]
            assert ctx.L.b200enc_ctx_device_outputs(ctypes.byref(ctx.ctx), *[ctypes.byref(p) for p in ptrs]) == 0
            mbs = ((w + 15) // 16) * ((h + 15) // 16)
            rd = lambda p, n: gpu.device_view(p.value, n).cpu().numpy()
            per.append({"levels": rd(ptrs[0], mbs * 768).view(np.int16).reshape(mbs, 24, 16),
                        "dc": rd(ptrs[1], mbs * 96).view(np.int32).reshape(mbs, 24),
                        "nz": rd(ptrs[2], mbs * 96).view(np.uint32).reshape(mbs, 24),
                        "pred_mode": rd(ptrs[3], mbs * 4).view(np.uint32),
                        "mv": rd(ptrs[4], mbs * 16).view(np.int32).reshape(mbs, 4),
                        "rec_y": y.copy(), "rec_uv": uv.copy()})
        ctx.close()
        res.append(per)
    return res


@pytest.mark.parametrize("me_mode,graph", [(0, False), (0, True), (3, False), (3, True)])
def test_batch_equals_single_stream_contexts(gpu, me_mode, graph):
    frames = _frames(gpu)
    want = _single(gpu, frames, me_mode)
    b = gpu.Batch(SIZES, search_range=32, me_mode=me_mode, deblock=1, graph=graph)
    try:
        for t in range(STEPS):
            b.encode([frames[s][t] for s in range(len(SIZES))], QPS, [_intra(s, t) for s in range(len(SIZES))])
            assert b.sync() == 0
            for s in range(len(SIZES)):
                got = b.outputs_host(s)
                for k in ("levels", "dc", "nz", "pred_mode", "mv", "rec_y", "rec_uv"):
                    np.testing.assert_array_equal(got[k], want[s][t][k], err_msg=f"step {t} stream {s} {SIZES[s]} {k}")
        if graph:
            inst, upd = b.graph_stats()
            assert inst + upd == STEPS and upd >= 1, (inst, upd)
    finally:
        b.close()


def test_batch_rejects_bad_steps(gpu):
    import torch
    b = gpu.Batch([(64, 48), (32, 32)])
    try:
        f = [gpu.NV12(64, 48), gpu.NV12(32, 32)]
        with pytest.raises(RuntimeError):
            b.encode(f, [26, 26], [True, False])  # a stream must start intra
        with pytest.raises(RuntimeError):
            b.encode(f, [26, 60], [True, True])   # QP out of range
        b.encode(f, [26, 30], [True, True])
        assert b.sync() == 0
        b.encode(f, [26, 30], [False, True])
        assert b.sync() == 0
        torch.cuda.synchronize()
    finally:
        b.close()
    assert gpu.lib().b200enc_batch_create(0, None, None, 32, 0, 0.9, 1) is None
