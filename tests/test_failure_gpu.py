"""Failure detection on the GPU without a GPU fault: the bounded wait that
every tensor-core pipeline stage uses gives up on an mbarrier that nothing
completes, reports AB_ERR_TIMEOUT through device memory, and leaves the
context usable (a GEMM right after it is correct)."""
import pytest
import torch

from augurv2_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_the_context_survives():
    L = N.lib()
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    cycles = torch.zeros(1, dtype=torch.int64, device="cuda")
    limit = 20_000_000                      # ~10 ms at the SM clock
    N.check(L.ab_tc_wait_probe(limit, N.ptr(status), N.ptr(cycles), N.stream_ptr()), "ab_tc_wait_probe")
    torch.cuda.synchronize()
    assert int(status.item()) == N.AB_ERR_TIMEOUT
    assert limit <= int(cycles.item()) < 4 * limit
    # the same context still runs the tensor-core pipeline correctly
    torch.manual_seed(0)
    A = torch.randn(256, 512, device="cuda").to(torch.bfloat16)
    B = torch.randn(128, 512, device="cuda").to(torch.bfloat16)
    C = torch.full((256, 128), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    N.check(L.ab_tc_gemm_bf16(256, 128, 512, N.ptr(A), 512, N.ptr(B), 512, N.ptr(C), 128, 1, N.ptr(err),
                              N.stream_ptr()), "gemm")
    torch.cuda.synchronize()
    assert int(err.item()) == N.AB_OK
    ref = A.float() @ B.float().t()
    scale = A.float().abs() @ B.float().abs().t()
    assert ((C - ref).abs() <= 1e-5 * scale + 1e-6).all()


def test_wait_probe_refuses_bad_arguments():
    L = N.lib()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    cycles = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert L.ab_tc_wait_probe(0, N.ptr(status), N.ptr(cycles), N.stream_ptr()) == N.AB_ERR_ARG
    assert L.ab_tc_wait_probe(10**12, N.ptr(status), N.ptr(cycles), N.stream_ptr()) == N.AB_ERR_ARG
    assert L.ab_tc_wait_probe(1000, None, N.ptr(cycles), N.stream_ptr()) == N.AB_ERR_ARG
