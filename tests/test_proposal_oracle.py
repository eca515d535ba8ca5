"""CPU checks of the proposal network's oracle and host-side helpers: the
oracle's backward pass against central finite differences (FP64), the Morton
row layout against a direct image-grid convolution, BF16 rounding, and the
checkpoint format."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import proposal_ref as pr  # noqa: E402


def _rand_params(rs, scale=0.3):
    n = sum(o * i + o for i, o in pr.LAYERS)
    return rs.standard_normal(n) * scale


def test_bf16_rounding_matches_torch():
    import torch
    rs = np.random.Generator(np.random.PCG64(3))
    x = np.concatenate([rs.standard_normal(10000).astype(np.float32) * 100,
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e-39, -7.5e-41, 65504.0], np.float32)])
    want = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(pr.bf16(x), want)


def test_morton_rows_are_a_grid_convolution():
    """Each 2x2 stride-2 layer as a GEMM over Morton rows equals the same
    convolution evaluated on the image grid."""
    rs = np.random.Generator(np.random.PCG64(5))
    img = rs.standard_normal((16, 16, 2))
    rows = np.zeros((64, 8))
    for m in range(64):
        ox, oy = pr.morton_xy(m)
        for dy in range(2):
            for dx in range(2):
                rows[m, (dy * 2 + dx) * 2:(dy * 2 + dx) * 2 + 2] = img[2 * oy + dy, 2 * ox + dx]
    grid, a = img, rows
    for l in range(4):
        W = rs.standard_normal((32, pr.LAYERS[l][0]))
        n = grid.shape[0] // 2
        direct = np.zeros((n, n, 32))
        for oy in range(n):
            for ox in range(n):
                patch = np.concatenate([grid[2 * oy + dy, 2 * ox + dx] for dy in range(2) for dx in range(2)])
                direct[oy, ox] = W @ patch
        gemm = a @ W.T  # rows in Morton order over the n x n grid
        for m in range(n * n):
            ox = (m & 1) | ((m >> 1) & 2) | ((m >> 2) & 4)
            oy = ((m >> 1) & 1) | ((m >> 2) & 2) | ((m >> 3) & 4)
            np.testing.assert_allclose(gemm[m], direct[oy, ox], rtol=1e-12, atol=1e-12)
        if l < 3:
            grid, a = direct, gemm.reshape(-1, 128)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_backward_matches_finite_differences(seed):
    rs = np.random.Generator(np.random.PCG64(seed))
    B = 3
    params = _rand_params(rs)
    x0 = rs.standard_normal((B * 64, 8))
    side = rs.standard_normal((B, 64))
    label = np.array([0b1, 0b10000000000, 0b1001000], np.int32)
    norez = np.array([1.0, 0.0, 1.0])
    weight = np.array([1.0, 1.0, 0.0])
    dup = np.array([0b10, 0, 0b1000000000])

    def loss_of(p):
        z, _ = pr.forward(p, x0, side, exact=True)
        return pr.loss_and_grad(z, label, norez, weight, dup)[0]

    z, acts = pr.forward(params, x0, side, exact=True)
    _, g5 = pr.loss_and_grad(z, label, norez, weight, dup)
    grad = pr.backward(params, acts, g5, exact=True)
    idx = rs.choice(params.size, 80, replace=False)
    # every layer's weights and biases are sampled
    offs, o = [], 0
    for i, n in pr.LAYERS:
        offs += [o, o + n * i]
        o += n * i + n
    idx = np.concatenate([idx, np.array(offs)])
    eps = 1e-6
    for k in idx:
        p1, p2 = params.copy(), params.copy()
        p1[k] += eps
        p2[k] -= eps
        fd = (loss_of(p1) - loss_of(p2)) / (2 * eps)
        assert abs(fd - grad[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, grad[k])


def test_loss_gradient_rows_sum_to_zero_over_classes():
    """Softmax CE: each weighted row's class gradient sums to zero and masked
    (duplicate) classes get none."""
    rs = np.random.Generator(np.random.PCG64(9))
    z = rs.standard_normal((5, 16))
    dup = np.array([0, 0b110, 0, 0b1000000000, 0])
    _, g = pr.loss_and_grad(z, np.array([1, 0b1001, 1 << 10, 1 << 4, 1 << 9 | 1]), np.zeros(5), np.ones(5), dup)
    np.testing.assert_allclose(g[:, :11].sum(axis=1), 0, atol=1e-12)
    assert g[1, 1] == 0 and g[1, 2] == 0 and g[3, 9] == 0


def test_checkpoint_roundtrip_and_hash(tmp_path):
    from b200enc import proposal
    p = proposal.init_params(7)
    assert p.size == proposal.NUM_PARAMS == sum(o * i + o for i, o in pr.LAYERS)
    path = str(tmp_path / "w.b2pn")
    proposal.save_checkpoint(path, p, step=12, meta={"qp": [22, 27]}, adam_m=p * 0, adam_v=p * 0 + 1)
    q, step, meta, adam = proposal.load_checkpoint(path)
    np.testing.assert_array_equal(p, q)
    assert step == 12 and meta == {"qp": [22, 27]} and adam[1][0] == 1
    data = bytearray(open(path, "rb").read())
    data[100] ^= 1
    open(path, "wb").write(bytes(data))
    with pytest.raises(ValueError):
        proposal.load_checkpoint(path)


def test_prepare_oracle_candidates_and_features():
    """Hand-checkable case: uniform previous motion gives two distinct
    candidates (the motion and zero) and the duplicate flags say so."""
    W, H = 48, 32
    rs = np.random.Generator(np.random.PCG64(1))
    ref = rs.integers(0, 256, (H, W), dtype=np.uint8)
    cur = np.roll(ref, (1, 2), axis=(0, 1))  # content moved by (+2, +1): MV (-2, -1)
    prev = np.zeros((6, 4), np.int32)
    prev[:, 0], prev[:, 1] = -8, -4
    d = pr.prepare(cur, ref, W, H, W, H, prev, 16, 512)
    assert (d["cand"][:, :9] == np.array([-2, -1])).all() and (d["cand"][:, 9] == 0).all()
    assert (d["state"] >> 8 == 0b111111110).all()
    # interior MB: zero SAD at the true motion
    assert d["cand_sad"][4, 0] == 0
    dn = pr.prepare(cur, ref, W, H, W, H, None, 16, 512)
    assert (dn["state"] & 2).all() and (dn["side"][:, 63] == 1).all()


def test_fp8_oracle_rounding_and_closeness():
    """E4M3 known answers (nearest-even, saturation at 448, subnormals down to
    2^-9) and the FP8 forward against the BF16 forward on random
    parameters: same top-1 class on >= 95 % of MBs, logits within 10 % of
    their spread."""
    v = np.array([0.5, 448.0, 500.0, -1000.0, 0.3, 1e-4, 0.0017578125, 17.0, 19.0], np.float32)
    np.testing.assert_array_equal(pr.e4m3(v), np.array([0.5, 448, 448, -448, 0.3125, 0, 2.0 ** -9, 16, 20],
                                                       np.float32))
    rs = np.random.default_rng(3)
    p = (rs.standard_normal(sum(i * o + o for i, o in pr.LAYERS)) * 0.1).astype(np.float32)
    B = 40  # 3 tiles, the last one partial
    x0 = rs.standard_normal((B * 64, 8)).astype(np.float32)
    side = (rs.standard_normal((B, 64)) * 0.5).astype(np.float32)
    lb, _ = pr.forward(p, x0, side)
    l8 = pr.forward_fp8(p, x0, side)
    spread = np.abs(lb).max()
    assert np.abs(lb - l8).max() <= 0.1 * spread
    assert (lb[:, :11].argmax(1) == l8[:, :11].argmax(1)).mean() >= 0.95
