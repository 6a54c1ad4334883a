"""Tensor-core GEMM and training kernels of the warm-start surrogate against float32 references.

The GEMM multiplies BF16 operands with FP32 accumulation, so the reference is a float32
matmul of the same BF16-rounded inputs; products of two BF16 numbers are exact in FP32 and
only the summation order differs, bounded by K * eps32 * sum |a_ik b_jk|.
"""

import numpy as np
import pytest
import torch

from snoopy_b200 import _lib

pytestmark = pytest.mark.gpu


def _p(t):
    return _lib.ptr(t) if t is not None else None


def gemm(A, B, bias=None, act=0, want_c=True, want_h=False):
    M, K = A.shape
    N = B.shape[0]
    C = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda") if want_c else None
    H = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda") if want_h else None
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("snp_gemm_bf16", M, N, K, _p(A), A.stride(0), _p(B), B.stride(0), _p(bias), act, _p(C), N,
              _p(H), N, _p(err), _lib.stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C, H


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (200, 256, 256), (300, 128, 256), (4000, 256, 16),
                                   (256, 16, 4000), (130, 48, 72), (1, 16, 8), (777, 300, 520)])
def test_gemm_bf16_matches_fp32(M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C, _ = gemm(A, B)
    ref = A.float() @ B.float().T
    scale = A.float().abs() @ B.float().abs().T
    err = ((C - ref).abs() / (scale + 1e-30)).max().item()
    assert err <= 4 * K * 2 ** -24 + 1e-7, err


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 300, 520), (1, 16, 8), (4000, 256, 16), (256, 16, 4000)])
def test_gemm_tma_pipeline_equals_plain_loads(M, N, K):
    """The TMA-fed, double-buffered kernel (default) and the kernel that stages operands with
    plain loads (SNP_GEMM_TMA=0) issue the same MMAs on the same shared-memory layout: the
    results are bitwise equal, boundary tiles (zero-filled by the TMA unit) included."""
    import os

    g = torch.Generator(device="cuda").manual_seed(M + 5 * N + 11 * K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    C1, H1 = gemm(A, B, bias=bias, act=1, want_h=True)
    os.environ["SNP_GEMM_TMA"] = "0"
    try:
        C0, H0 = gemm(A, B, bias=bias, act=1, want_h=True)
    finally:
        del os.environ["SNP_GEMM_TMA"]
    assert torch.equal(C1, C0) and torch.equal(H1, H0)


def test_gemm_bias_gelu_epilogue():
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(384, 256, device="cuda", generator=g).to(torch.bfloat16)
    B = (0.05 * torch.randn(128, 256, device="cuda", generator=g)).to(torch.bfloat16)
    bias = torch.randn(128, device="cuda", generator=g)
    C, H = gemm(A, B, bias=bias, act=1, want_h=True)
    Z = A.float() @ B.float().T + bias
    assert torch.allclose(C, Z, rtol=1e-4, atol=1e-4)
    Hf = 0.5 * Z * (1 + torch.erf(Z / np.sqrt(2.0)))
    assert torch.allclose(H.float(), Hf, rtol=1e-2, atol=1e-2)  # BF16 output rounding


def test_gemm_rejects_bad_shapes():
    A = torch.zeros(128, 12, dtype=torch.bfloat16, device="cuda")
    B = torch.zeros(16, 12, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    C = torch.zeros(128, 16, device="cuda")
    rc = _lib.load().snp_gemm_bf16(128, 16, 12, _p(A), 12, _p(B), 12, None, 0, _p(C), 16, None, 16, _p(err),
                                   _lib.stream_ptr())
    assert rc != 0 and b"multiple of 8" in _lib.load().snp_last_error()


def test_elementwise_training_kernels():
    g = torch.Generator(device="cuda").manual_seed(5)
    Z = torch.randn(1000, device="cuda", generator=g)
    dH = torch.randn(1000, device="cuda", generator=g)
    dZ = torch.zeros(1000, device="cuda")
    _lib.call("snp_gelu_backward", 1000, _p(dH), _p(Z), None, _p(dZ), _lib.stream_ptr())
    Zr = Z.detach().clone().requires_grad_(True)
    (0.5 * Zr * (1 + torch.erf(Zr / np.sqrt(2.0)))).backward(dH)
    assert torch.allclose(dZ, Zr.grad, rtol=1e-5, atol=1e-6)

    X = torch.randn(70, 45, device="cuda", generator=g).to(torch.bfloat16)
    XT = torch.zeros(45, 70, dtype=torch.bfloat16, device="cuda")
    _lib.call("snp_transpose_bf16", 70, 45, _p(X), 45, _p(XT), 70, _lib.stream_ptr())
    assert torch.equal(XT, X.T)

    Y = torch.randn(300, 40, device="cuda", generator=g)
    s = torch.zeros(40, device="cuda")
    _lib.call("snp_col_sum", 300, 40, _p(Y), 40, _p(s), _lib.stream_ptr())
    assert torch.allclose(s, Y.sum(0), rtol=1e-5, atol=1e-4)

    w = torch.randn(500, device="cuda", generator=g)
    grad = torch.randn(500, device="cuda", generator=g)
    m = torch.zeros(500, device="cuda")
    v = torch.zeros(500, device="cuda")
    wb = torch.zeros(500, dtype=torch.bfloat16, device="cuda")
    ref = w.clone()
    mr, vr = torch.zeros_like(w), torch.zeros_like(w)
    for step in (1, 2, 3):
        _lib.call("snp_adam_step", 500, _p(w), _p(grad), _p(m), _p(v), _p(wb), 1e-3, 0.9, 0.999, 1e-8, step,
                  _lib.stream_ptr())
        mr = 0.9 * mr + 0.1 * grad
        vr = 0.999 * vr + 0.001 * grad * grad
        ref = ref - 1e-3 * (mr / (1 - 0.9 ** step)) / (torch.sqrt(vr / (1 - 0.999 ** step)) + 1e-8)
    torch.cuda.synchronize()
    assert torch.allclose(w, ref, rtol=1e-5, atol=1e-6)
    assert torch.equal(wb, w.to(torch.bfloat16))


def test_basis_combine_matches_float64_reference():
    """The POD reconstruction kernel (snp_basis_combine) against a float64 torch statement of
    mean + coef @ V^T with the same float32 basis: within 1e-13 of the result's scale, for
    several vector counts and basis widths (including P > 32, split into launches)."""
    import torch

    from snoopy_b200.surrogate import basis_combine

    g = torch.Generator(device="cuda").manual_seed(0)
    for n, m, P in ((1000, 128, 1), (70001, 128, 8), (5003, 64, 40), (777, 5, 3)):
        V = torch.randn((n, m), generator=g, device="cuda", dtype=torch.float32)
        c = torch.randn((P, m), generator=g, device="cuda", dtype=torch.float64)
        mean = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
        got = basis_combine(V, c, mean)
        want = mean + c @ V.double().T
        assert float((got - want).abs().max() / want.abs().max()) < 1e-13, (n, m, P)
        got0 = basis_combine(V, c)
        assert float((got0 - (c @ V.double().T)).abs().max() / want.abs().max()) < 1e-13
