"""The autotuner's launch shapes change no result: every candidate value of
every knob (deblocking rows per CTA, P-chain macroblocks per CTA, the
re-scoring and fallback grids, the intra wavefront's CTA count, the full
search's window staging by TMA or by loads, the deblocking tile's width and
height) gives the
default's staged outputs and reconstruction bit for bit, on the learned form
at 1920x1080 (I frame, a full-search P frame, learned P frames); and the
tuner's choice is one of the candidates and is applied to the table."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, QP = 1920, 1080, 30


def _frames(gpu, n=4):
    from b200enc import synth
    seq = synth.workload("h264_1080p", seed=0, stream=77)
    return [gpu.NV12.from_host(*seq.frame(t)) for t in range(n)]


def _encode(gpu, frames):
    ctx = gpu.Context()
    ctx.configure(search_range=32, lam=5, zero_thresh=512, coded_clamp=True, deblock=1)
    ctx.set_me(3)
    out = []
    for t, fr in enumerate(frames):
        ctx.encode_device(fr, W, H, QP, t == 0, 1, False)
        y, uv = ctx.recon_host()
        mv = ctx.mv_field()
        lev, dc, nz, pm, _ = (gpu.device_view(p, n).cpu().numpy().copy() for p, n in _outputs(gpu, ctx))
        out.append((y.copy(), uv.copy(), mv.copy(), lev, dc, nz, pm))
    ctx.close()
    return out


def _outputs(gpu, ctx):
    import ctypes
    ptrs = [ctypes.c_void_p() for _ in range(5)]
    assert ctx.L.b200enc_ctx_device_outputs(ctypes.byref(ctx.ctx), *[ctypes.byref(p) for p in ptrs]) == 0
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    sizes = [mbs * 768, mbs * 96, mbs * 96, mbs * 4, mbs * 16]
    return [(p.value, n) for p, n in zip(ptrs, sizes)]


def test_every_knob_value_is_exact(gpu):
    from b200enc import autotune
    frames = _frames(gpu)
    autotune.apply({k: 0 for k in autotune.KEYS})
    want = _encode(gpu, frames)
    mbh = (H + 15) // 16
    try:
        for name in autotune.KEYS:
            for v in autotune.candidates(name, mbh):
                autotune.apply({name: v})
                got = _encode(gpu, frames)
                for t, (g, w) in enumerate(zip(got, want)):
                    for k, (a, b) in enumerate(zip(g, w)):
                        np.testing.assert_array_equal(a, b, err_msg=f"{name}={v} frame {t} output {k}")
            autotune.apply({name: 0})
    finally:
        autotune.apply({k: 0 for k in autotune.KEYS})


def test_tuner_picks_a_candidate(gpu, tmp_path):
    from b200enc import autotune
    frames = _frames(gpu, 5)
    try:
        vals, src, _ = autotune.load_or_tune(frames, W, H, cache=str(tmp_path / "tune.json"), reps=1)
        assert src == "tuned"
        mbh = (H + 15) // 16
        for name in autotune.TUNED:  # deblock_rows (the stage-level wavefront's) stays at its default
            assert vals[name] in autotune.candidates(name, mbh), (name, vals[name])
        assert vals["deblock_rows"] == 0
        assert autotune.current() == vals
        again, src2, _ = autotune.load_or_tune(frames, W, H, cache=str(tmp_path / "tune.json"))
        assert src2 == "cache" and again == vals
    finally:
        autotune.apply({k: 0 for k in autotune.KEYS})
