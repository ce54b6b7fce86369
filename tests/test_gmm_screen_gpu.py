"""The Gaussian-mixture assignment draw screened in binary32
(ab_gmm_disc_z_screened) gives the reference's draw bit for bit: equal to the
binary64 kernel (ab_gmm_disc_z, itself equal to the FP64 oracle of
augur_mvnormal_ll + augur_unnorm_disc_samp, tests/test_gmm_gpu.py) on every
point, on the benchmark shape and on shapes that exercise the exact path
(zero weights, points far from every component, extreme log-densities, equal
components, shapes outside the screen's limits)."""
import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _draws(Y, pis, mus, covs, shared, seed=4, it=6):
    L = N.lib()
    N_, d = Y.shape
    K = len(pis)
    Kc = 1 if shared else K
    dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dt)
    Yd = dev(Y, torch.float32)
    cov = dev(covs[:Kc], torch.float64)
    Linv = torch.zeros((Kc, d, d), dtype=torch.float64, device="cuda")
    hdet = torch.zeros(Kc, dtype=torch.float64, device="cuda")
    N.check(L.ab_gmm_prep(Kc, d, N.ptr(cov), N.ptr(Linv), N.ptr(hdet), N.stream_ptr()), "prep")
    pd, md = dev(pis, torch.float64), dev(mus, torch.float64)
    z0 = torch.full((N_,), -1, dtype=torch.int32, device="cuda")
    z1 = torch.full((N_,), -1, dtype=torch.int32, device="cuda")
    N.check(L.ab_gmm_disc_z(N_, d, K, int(shared), N.ptr(Yd), N.ptr(pd), N.ptr(md), N.ptr(Linv), N.ptr(hdet),
                            N.ptr(z0), seed, it, 0, N.stream_ptr()), "disc_z")
    scratch = torch.zeros(int(L.ab_gmm_z_scratch_bytes(N_, d, K)), dtype=torch.uint8, device="cuda")
    N.check(L.ab_gmm_disc_z_screened(N_, d, K, int(shared), N.ptr(Yd), N.ptr(pd), N.ptr(md), N.ptr(Linv),
                                     N.ptr(hdet), N.ptr(z1), seed, it, 0, N.ptr(scratch), N.stream_ptr()),
            "disc_z_screened")
    torch.cuda.synchronize()
    return z0.cpu().numpy(), z1.cpu().numpy(), scratch


def _queued(scratch, d, K):
    """Points the screen left to the binary64 path (the queue length)."""
    off = int(N.lib().ab_gmm_z_queue_offset(d, K))
    return int(scratch[off:off + 4].view(torch.int32).item())


def test_screen_equals_binary64_on_the_benchmark_shape():
    N_, K, d = 200_000, 16, 32
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, 0)
    a, b, scratch = _draws(Y, pis, mus, covs, False)
    np.testing.assert_array_equal(b, a)
    q = _queued(scratch, d, K)
    assert q < N_ // 100, q            # the screen decides almost every point


@pytest.mark.parametrize("N_,K,d,shared,seed", [(5000, 4, 5, False, 1), (3000, 1, 3, False, 2),
                                                (4000, 32, 8, True, 3), (2500, 7, 2, False, 4),
                                                (1000, 16, 33, False, 5), (3000, 33, 4, False, 6)])
def test_screen_equals_binary64(N_, K, d, shared, seed):
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, seed)
    a, b, _ = _draws(Y, pis, mus, covs, shared, seed=seed)
    np.testing.assert_array_equal(b, a)


def test_screen_exact_path_cases():
    rng = np.random.default_rng(7)
    N_, K, d = 4000, 6, 6
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, 7)
    # zero weights; two equal components (ties at every point)
    pis = pis.copy()
    pis[1] = 0.0
    mus[3], covs[3] = mus[2], covs[2]
    pis = pis / pis.sum()
    Y = Y.copy()
    Y[:50] = 1e4 * rng.standard_normal((50, d))        # far from every component
    a, b, _ = _draws(Y, pis, mus, covs, False, seed=7)
    np.testing.assert_array_equal(b, a)
    # a tiny covariance: c - hdet > 700, every point takes the binary64 path
    covs2 = covs.copy()
    covs2[0] = 1e-300 * np.eye(d)
    a, b, scratch = _draws(Y, pis, mus, covs2, False, seed=8)
    np.testing.assert_array_equal(b, a)
    assert _queued(scratch, d, K) == N_
