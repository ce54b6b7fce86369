"""The tcgen05/TMA GEMM core against a float32 matrix product of the same
bf16 inputs (products are exact in FP32; only the summation order differs,
so agreement is to FP32 rounding: 1e-5 of the absolute-value product)."""
import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,Nn,K,splits", [(256, 256, 512, 1), (300, 100, 200, 1), (128, 64, 64, 1),
                                           (1000, 512, 768, 1), (256, 256, 4096, 4), (77, 33, 136, 2)])
def test_gemm_matches_fp32_reference(M, Nn, K, splits):
    torch.manual_seed(M + Nn + K)
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    B = torch.randn(Nn, K, device="cuda").to(torch.bfloat16)
    C = torch.full((M, Nn), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    N.check(N.lib().ab_tc_gemm_bf16(M, Nn, K, N.ptr(A), K, N.ptr(B), K, N.ptr(C), Nn, splits, N.ptr(err),
                                    N.stream_ptr()), "gemm")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.float() @ B.float().t()
    scale = A.float().abs() @ B.float().abs().t()
    assert torch.isfinite(C).all()
    assert ((C - ref).abs() <= 1e-5 * scale + 1e-6).all(), float(((C - ref).abs() / (scale + 1e-6)).max())


def test_gemm_rejects_unaligned_rows():
    A = torch.zeros(8, 130, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(8, 8, device="cuda")
    rc = N.lib().ab_tc_gemm_bf16(8, 8, 130, N.ptr(A), 130, N.ptr(A), 130, N.ptr(C), 8, 1, None, N.stream_ptr())
    assert rc != 0 and "16 bytes" in N.last_error()
