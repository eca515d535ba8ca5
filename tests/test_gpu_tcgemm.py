"""The tcgen05 BF16 GEMM (b200enc_gemm_bf16) against an FP64 product of the
same BF16 values.

Tolerance: each output may differ from the exact sum by at most
1e-4 x sum_k |A(m,k) B(n,k)| + 1e-6 (FP32 accumulation over at most a few
thousand terms; BF16 x BF16 products are exact in FP32).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16(rs, shape, scale=1.0):
    import torch
    return (torch.from_numpy(rs.standard_normal(shape).astype(np.float32)) * scale).to(torch.bfloat16)


def _check(got, A, B, C0, bias, flags):
    a = A.double()
    b = B.double()
    want = a @ b.T
    bound = a.abs() @ b.abs().T
    if flags & 1:
        want = want + C0.double()
        bound = bound + C0.double().abs()
    if bias is not None:
        want = want + bias.double()[None, :]
        bound = bound + bias.double().abs()[None, :]
    if flags & 2:
        want = want.clamp_min(0)
    err = (got.double() - want).abs()
    tol = 1e-4 * bound + 1e-6
    bad = err > tol
    assert not bad.any(), f"{int(bad.sum())} outputs off; worst {float((err - tol).max())}"


SHAPES = [(1, 1, 1), (128, 32, 64), (200, 50, 100), (129, 65, 16), (300, 128, 700), (1000, 200, 300),
          (64, 17, 1000), (4096, 96, 288), (513, 304, 160)]


@pytest.mark.parametrize("M,N,K", SHAPES)
@pytest.mark.parametrize("layout", ["nt", "tn", "tt"])
def test_gemm_bf16(gpu, M, N, K, layout):
    import torch
    rs = np.random.Generator(np.random.PCG64(M * 7 + N * 3 + K))
    A = _bf16(rs, (M, K))
    B = _bf16(rs, (N, K))
    # operand storage: "n" = K-contiguous rows, "t" = stored transposed (rows contiguous)
    Ad = (A.cuda().contiguous() if layout[0] == "n" else A.T.contiguous().cuda())
    Bd = (B.cuda().contiguous() if layout[1] == "t" else B.T.contiguous().cuda())
    a_str = (K, 1) if layout[0] == "n" else (1, M)
    b_str = (K, 1) if layout[1] == "t" else (1, N)
    C = torch.full((M, N + 3), float("nan"), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    gpu.gemm_bf16(Ad, Bd, C, M, N, K, a_str, b_str, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    _check(C[:, :N].cpu(), A, B, None, None, 0)
    assert torch.isnan(C[:, N:]).all(), "wrote outside the N columns"


@pytest.mark.parametrize("flags", [1, 2, 3])
@pytest.mark.parametrize("with_bias", [False, True])
def test_gemm_bf16_epilogue(gpu, flags, with_bias):
    import torch
    M, N, K = 333, 72, 200
    rs = np.random.Generator(np.random.PCG64(flags * 10 + with_bias))
    A, B = _bf16(rs, (M, K)), _bf16(rs, (N, K))
    C0 = torch.from_numpy(rs.standard_normal((M, N)).astype(np.float32)) * 5
    bias = torch.from_numpy(rs.standard_normal(N).astype(np.float32)) if with_bias else None
    C = C0.cuda()
    gpu.gemm_bf16(A.cuda(), B.cuda(), C, M, N, K, (K, 1), (K, 1), bias=bias.cuda() if with_bias else None,
                  flags=flags)
    torch.cuda.synchronize()
    _check(C.cpu(), A, B, C0, bias, flags)


@pytest.mark.parametrize("M,N,K", [(300, 32, 8), (1000, 64, 128), (513, 96, 40)])
@pytest.mark.parametrize("relu", [False, True])
def test_gemm_bf16_out(gpu, M, N, K, relu):
    """BF16 output: the FP32 result (bias, ReLU) rounded to nearest even."""
    import torch
    rs = np.random.Generator(np.random.PCG64(M + N + K + relu))
    A, B = _bf16(rs, (M, K)), _bf16(rs, (N, K))
    bias = torch.from_numpy(rs.standard_normal(N).astype(np.float32))
    C = torch.zeros((M, N + 8), dtype=torch.bfloat16, device="cuda")
    gpu.gemm_bf16(A.cuda(), B.cuda(), C, M, N, K, (K, 1), (K, 1), bias=bias.cuda(),
                  flags=gpu.GEMM_OUT_BF16 | (gpu.GEMM_RELU if relu else 0))
    torch.cuda.synchronize()
    want = A.double() @ B.double().T + bias.double()[None, :]
    if relu:
        want = want.clamp_min(0)
    got = C[:, :N].cpu().double()
    # one BF16 rounding of a value within the FP32 tolerance of the exact sum
    bound = A.double().abs() @ B.double().abs().T + bias.double().abs()[None, :]
    err = (got - want).abs()
    tol = 2.0 ** -8 * want.abs() + 1e-4 * bound + 1e-6
    assert (err <= tol).all()
    assert (C[:, N:].cpu() == 0).all()


@pytest.mark.parametrize("M,N,K,splits", [(32, 128, 100000, 37), (128, 288, 5000, 8), (64, 17, 700, 3),
                                          (32, 32, 64, 5)])
def test_gemm_bf16_splitk(gpu, M, N, K, splits):
    """Split K: slices add into C atomically (C += A.B^T), including slices
    that own no K chunk."""
    import torch
    rs = np.random.Generator(np.random.PCG64(K + splits))
    A, B = _bf16(rs, (M, K)), _bf16(rs, (N, K))
    C0 = torch.from_numpy(rs.standard_normal((M, N)).astype(np.float32))
    C = C0.cuda()
    # transposed storage of A exercises strided staging too
    Ad = A.T.contiguous().cuda()
    gpu.gemm_bf16(Ad, B.cuda(), C, M, N, K, (1, M), (K, 1), flags=gpu.GEMM_SPLITK(splits))
    torch.cuda.synchronize()
    _check(C.cpu(), A, B, C0, None, 1)


def test_gemm_bf16_rejects_bad_splitk(gpu):
    import torch
    A = torch.zeros((128, 64), dtype=torch.bfloat16, device="cuda")
    C = torch.zeros((128, 64), dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError):
        gpu.gemm_bf16(A, A, C, 128, 64, 64, (64, 1), (64, 1), flags=gpu.GEMM_SPLITK(4) | gpu.GEMM_RELU)
