"""The learned motion-proposal network: parameter layout, checkpoints and the
runtime handle of libb200enc.so (csrc/proposal.cu). Every forward, backward
and optimizer step runs in the library's CUDA kernels on the tcgen05 tensor
cores; this module only allocates, loads and drives them.

Network (per 16x16 MB; rows of the conv layers in Morton order):
  input   [64 rows][8]   2x2 pels x (current luma, residual at candidate 0)
  conv1   8 -> 32        2x2 stride 2, 16x16 -> 8x8      (a GEMM over rows)
  conv2   128 -> 32      2x2 stride 2, 8x8 -> 4x4
  conv3   128 -> 32      2x2 stride 2, 4x4 -> 2x2
  conv4   128 -> 32      2x2 stride 2, 2x2 -> 1x1
  fc1     96 -> 64       conv features + 64 side features
  fc2     64 -> 16       10 candidate logits, "none", no-residual, 4 unused
Parameters are stored layer by layer as W [out][in] (row-major) then b [out].
"""
import ctypes
import hashlib
import json
import os
import struct

import numpy as np

LAYERS = [(8, 32), (128, 32), (128, 32), (128, 32), (96, 64), (64, 16)]  # (in, out)
N_CAND, N_CLASSES, N_OUT, N_FEAT, F_IN = 10, 11, 16, 64, 96


def layer_offsets():
    """[(w_off, b_off, in, out)] of each layer in the flat parameter vector."""
    offs, o = [], 0
    for i, n in LAYERS:
        offs.append((o, o + n * i, i, n))
        o += n * i + n
    return offs


NUM_PARAMS = sum(n * i + n for i, n in LAYERS)

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "proposal_h264.b2pn")
_MAGIC = b"B2PN"


def init_params(seed=0):
    """He-uniform weights, zero biases; the output layer starts 10x smaller."""
    rs = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(NUM_PARAMS, np.float32)
    for li, (wo, bo, i, n) in enumerate(layer_offsets()):
        lim = np.sqrt(6.0 / i) * (0.1 if li == len(LAYERS) - 1 else 1.0)
        p[wo:bo] = rs.uniform(-lim, lim, n * i).astype(np.float32)
    return p


def save_checkpoint(path, params, step=0, meta=None, adam_m=None, adam_v=None):
    """Binary checkpoint: magic, version, n, step, meta JSON, params, optional
    Adam moments, then the SHA-256 of everything before it."""
    params = np.ascontiguousarray(params, np.float32)
    assert params.size == NUM_PARAMS
    mj = json.dumps(meta or {}, sort_keys=True).encode()
    has_adam = adam_m is not None and adam_v is not None
    body = _MAGIC + struct.pack("<IIIII", 1, NUM_PARAMS, int(step), len(mj), int(has_adam)) + mj + params.tobytes()
    if has_adam:
        body += np.ascontiguousarray(adam_m, np.float32).tobytes() + np.ascontiguousarray(adam_v, np.float32).tobytes()
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "wb") as f:
        f.write(body + hashlib.sha256(body).digest())
    return hashlib.sha256(body).hexdigest()


def load_checkpoint(path):
    """(params, step, meta, (adam_m, adam_v) or None); raises on a bad hash."""
    with open(path, "rb") as f:
        data = f.read()
    body, digest = data[:-32], data[-32:]
    if hashlib.sha256(body).digest() != digest:
        raise ValueError(f"{path}: checksum mismatch")
    if body[:4] != _MAGIC:
        raise ValueError(f"{path}: not a proposal checkpoint")
    ver, n, step, mlen, has_adam = struct.unpack("<IIIII", body[4:24])
    if ver != 1 or n != NUM_PARAMS:
        raise ValueError(f"{path}: version {ver} / {n} parameters, expected 1 / {NUM_PARAMS}")
    meta = json.loads(body[24:24 + mlen].decode())
    o = 24 + mlen
    params = np.frombuffer(body, np.float32, n, o).copy()
    adam = None
    if has_adam:
        m = np.frombuffer(body, np.float32, n, o + 4 * n).copy()
        v = np.frombuffer(body, np.float32, n, o + 8 * n).copy()
        adam = (m, v)
    return params, step, meta, adam


# tensor indices of b200enc_proposal_tensor
T_PARAMS, T_GRADS, T_X0, T_Y1, T_Y2, T_Y3, T_F, T_H, T_LOGITS, T_CAND, T_CAND_SAD, T_STATE, T_SEL, T_NOREZ, \
    T_LISTS, T_COUNTERS, T_LABEL, T_NOREZ_T, T_WEIGHT, T_LOSS, T_ERR = range(21)

_BF16 = "bf16"


class Proposal:
    """A runtime handle: parameters, activations for up to max_mbs MBs and,
    after the first training call, gradients and Adam state."""

    def __init__(self, max_mbs, params=None):
        from . import lib
        self._lib = lib()
        self.max_mbs = max_mbs
        self.h = self._lib.b200enc_proposal_create(max_mbs)
        if not self.h:
            raise RuntimeError("b200enc_proposal_create failed")
        if params is not None:
            self.set_params(params)

    def close(self):
        if self.h:
            self._lib.b200enc_proposal_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed (rc={rc})")

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        self._ck(self._lib.b200enc_proposal_set_params(self.h, p.ctypes.data, p.size), "set_params")

    def load(self, path):
        """Parameters from a checkpoint, read and SHA-256-checked by the library."""
        rc = self._lib.b200enc_proposal_load(self.h, os.fsencode(path))
        if rc != 0:
            raise RuntimeError(f"b200enc_proposal_load({path}) failed (rc={rc})")

    def get_params(self):
        p = np.zeros(NUM_PARAMS, np.float32)
        self._ck(self._lib.b200enc_proposal_get_params(self.h, p.ctypes.data, p.size), "get_params")
        return p

    def tensor(self, which, dtype, shape):
        """A torch view of an internal device tensor (no copy)."""
        import torch
        from . import device_view
        ptr, n = ctypes.c_void_p(), ctypes.c_size_t()
        self._ck(self._lib.b200enc_proposal_tensor(self.h, which, ctypes.byref(ptr), ctypes.byref(n)), "tensor")
        tdt = torch.bfloat16 if dtype == _BF16 else dtype
        count = int(np.prod(shape))
        esize = torch.empty((), dtype=tdt).element_size()
        assert count * esize <= n.value, (which, shape, n.value)
        return device_view(ptr.value, count * esize).view(tdt).view(*shape)

    def prepare(self, cur, ref, W, H, RW, RH, prev_mv, rng, zero_thresh, stream=None):
        from . import _p, _stream
        self._ck(self._lib.b200enc_proposal_prepare(self.h, cur.yp(), cur.pitch, ref.yp(), ref.pitch, W, H, RW, RH,
                                                    _p(prev_mv) if prev_mv is not None else None, rng, zero_thresh,
                                                    _stream(stream)), "prepare")

    def forward(self, mbs, stream=None):
        from . import _stream
        self._ck(self._lib.b200enc_proposal_forward(self.h, mbs, _stream(stream)), "forward")

    def labels(self, mbs, logged_mv, nz=None, stream=None):
        from . import _p, _stream
        self._ck(self._lib.b200enc_proposal_labels(self.h, mbs, _p(logged_mv), _p(nz) if nz is not None else None,
                                                   _stream(stream)), "labels")

    def backward(self, mbs, stream=None):
        from . import _stream
        self._ck(self._lib.b200enc_proposal_backward(self.h, mbs, _stream(stream)), "backward")

    def adam(self, lr, step, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        from . import _stream
        self._ck(self._lib.b200enc_proposal_adam(self.h, lr, beta1, beta2, eps, step, _stream(stream)), "adam")

    def train_step(self, mbs, lr, step, stream=None):
        from . import _stream
        self._ck(self._lib.b200enc_proposal_train_step(self.h, mbs, lr, step, _stream(stream)), "train_step")

    NETWORK, CANDIDATES, NETWORK_FP8 = 1, 2, 3

    def me(self, cur, ref, W, H, RW, RH, prev_mv, rng, lam, zero_thresh, param, mv_out, mode=1, stream=None):
        """Learned-form ME of one frame: mode NETWORK (param = confidence
        threshold), NETWORK_FP8 (the same with FP8 inference) or CANDIDATES
        (no network; param = fallback cost per pel, < 0 never)."""
        from . import _p, _stream
        self._ck(self._lib.b200enc_proposal_me(self.h, cur.yp(), cur.pitch, ref.yp(), ref.pitch, W, H, RW, RH,
                                               _p(prev_mv) if prev_mv is not None else None, rng, lam, zero_thresh,
                                               mode, param, _p(mv_out), _stream(stream)), "proposal_me")

    def counters(self):
        """[learned, fallback, valid training samples, early-outs] (synchronises)."""
        import torch
        torch.cuda.synchronize()
        return self.tensor(T_COUNTERS, torch.int32, (8,)).cpu().numpy()[:4].copy()
