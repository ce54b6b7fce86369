"""ab_lda_conj_phi_noalloc - the phi draw for callers that cannot allocate
device memory (a host framework that owns all device memory through its own
pool, or a plugin that must not allocate while it runs) - gives the same
result as ab_lda_conj_phi with a caller-allocated scratch buffer, on two
calls in a row, through the C ABI.  Kept last in collection order so a
failure here comes after every other test has run."""
import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N

pytestmark = pytest.mark.gpu
RTOL = 1e-12   # the tolerance of the other phi parity tests


def _inputs(K, V, seed):
    rng = np.random.default_rng(seed)
    cnt = torch.as_tensor(rng.poisson(1.0, size=(K, V)).astype(np.int32)).cuda()
    beta = torch.full((V,), 0.01, dtype=torch.float64, device="cuda")
    Kp = N.lib().ab_lda_phi_stride(K)
    return cnt, beta, Kp


def test_noalloc_matches_caller_scratch_twice():
    L = N.lib()
    K, V = 50, 10000
    for call, (seed, it) in enumerate([(3, 0), (4, 1)]):
        cnt, beta, Kp = _inputs(K, V, seed + 10 * call)
        cnt2 = cnt.clone()
        out_a = torch.zeros((V, Kp), dtype=torch.float64, device="cuda")
        out_b = torch.zeros((V, Kp), dtype=torch.float64, device="cuda")
        scratch = torch.zeros(int(L.ab_lda_phi_scratch_bytes(K, V)), dtype=torch.uint8, device="cuda")
        N.check(L.ab_lda_conj_phi(K, V, N.ptr(beta), N.ptr(cnt), N.ptr(out_a), 1, seed, it, N.ptr(scratch),
                                  N.stream_ptr()), "ab_lda_conj_phi")
        N.check(L.ab_lda_conj_phi_noalloc(K, V, N.ptr(beta), N.ptr(cnt2), N.ptr(out_b), 1, seed, it,
                                          N.stream_ptr()), "ab_lda_conj_phi_noalloc")
        torch.cuda.synchronize()
        a, b = out_a.cpu().numpy()[:, :K], out_b.cpu().numpy()[:, :K]
        # same kernels, same seed and counts: identical bits
        assert np.array_equal(b, a)
        np.testing.assert_allclose(b.sum(0), 1.0, rtol=RTOL)
        assert (cnt2.cpu().numpy() == 0).all()


def test_noalloc_rejects_sizes_beyond_the_builtin_scratch():
    L = N.lib()
    K, V = 1024, 300000          # needs about 9.6 MB of scratch
    assert L.ab_lda_phi_scratch_bytes(K, V) > (1 << 20)
    # valid pointers, so the refusal comes from the scratch-size check
    rc = L.ab_lda_conj_phi_noalloc(K, V, N.ptr(torch.zeros(1, device="cuda", dtype=torch.float64)),
                                   N.ptr(torch.zeros(1, device="cuda", dtype=torch.int32)),
                                   N.ptr(torch.zeros(1, device="cuda", dtype=torch.float64)), 0, 0, 0,
                                   N.stream_ptr())
    assert rc == 1 and "scratch" in N.last_error()
