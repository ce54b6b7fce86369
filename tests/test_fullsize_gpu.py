"""Parity at the benchmark shapes themselves.

* LDA at K=50, V=1e4, D=2000 with Poisson(200) document lengths (the Gibbs
  tokens/s workload): one ab_lda_disc_z call with both count tables, on the
  state a few sweeps produce, gives assignments and counts equal to the CPU
  oracle's bit for bit; one graph-replayed sweep of the sampler meets the
  per-sweep contract (theta and phi within 1e-12 of the oracle's draws from
  the previous sweep's counts, z bit-exact given them).
* Gaussian mixture at K=16, d=32, N=2e5: the assignment pass runs over all
  points on the device and every 10th point is checked bit for bit against
  the oracle (which re-factors each covariance per point and component as
  the reference does, so the full N would take minutes on one core); one
  full sweep meets the per-sweep contract at that size.
"""
import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N
from augurv2_b200.gmm import GmmGibbs
from augurv2_b200.lda import LdaGibbs, synthetic_corpus
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-12          # theta / phi against the oracle's gamma draws


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


@pytest.fixture(scope="module")
def lda_bench():
    K, V, D = 50, 10000, 2000
    off, w = synthetic_corpus(K, V, D, 200, 0.1, 0.01, seed=0)
    s = LdaGibbs(K, V, off, w, 0.1, 0.01, seed=1000)
    s.sweep(4)
    yield K, V, D, off, w, s
    s.close()


def test_lda_disc_z_and_counts_bit_exact_at_benchmark_shape(orc, lda_bench):
    K, V, D, off, w, s = lda_bench
    theta, phi, _ = s.state()
    z = torch.zeros(len(w), dtype=torch.int32, device="cuda")
    cdk = torch.full((D, K), -1, dtype=torch.int32, device="cuda")
    ckw = torch.zeros((K, V), dtype=torch.int32, device="cuda")
    seed, it = 77, 123
    N.check(N.lib().ab_lda_disc_z(D, K, V, N.ptr(s.doc_off), N.ptr(s.w), N.ptr(s.theta), N.ptr(s.phiT),
                                  N.ptr(z), N.ptr(cdk), N.ptr(ckw), seed, it, N.stream_ptr()), "disc_z")
    z_ref = orc.lda_disc_z(off, w, theta, phi, np.zeros(len(w), np.int32), seed, it)
    np.testing.assert_array_equal(z.cpu().numpy(), z_ref)
    c_dk, c_kw = orc.lda_conj_stat(off, w, z_ref, D, K, V)
    np.testing.assert_array_equal(cdk.cpu().numpy(), c_dk)
    np.testing.assert_array_equal(ckw.cpu().numpy(), c_kw)
    # the drawn state is not degenerate: most topics are used
    assert (c_dk.sum(0) > 0).sum() >= K // 2


def test_lda_sweep_per_sweep_contract_at_benchmark_shape(orc, lda_bench):
    K, V, D, off, w, s = lda_bench
    z_prev = s.state()[2]
    it = s.iteration
    s.sweep(1)
    theta, phi, z = s.state()
    alpha, beta = np.full(K, 0.1), np.full(V, 0.01)
    c_dk, c_kw = orc.lda_conj_stat(off, w, z_prev, D, K, V)
    np.testing.assert_allclose(theta, orc.lda_conj_theta(alpha, c_dk, s.seed, it), rtol=RTOL, atol=0)
    np.testing.assert_allclose(phi, orc.lda_conj_phi(beta, c_kw, s.seed, it), rtol=RTOL, atol=1e-300)
    z_ref = orc.lda_disc_z(off, w, theta, phi, np.zeros_like(z), s.seed, it)
    np.testing.assert_array_equal(z, z_ref)
    # the counts the sampler holds for the next sweep are those of the new z
    c_dk, c_kw = orc.lda_conj_stat(off, w, z, D, K, V)
    np.testing.assert_array_equal(s.cnt_dk.cpu().numpy(), c_dk)
    np.testing.assert_array_equal(s.cnt_kw.cpu().numpy(), c_kw)


GMM_K, GMM_D, GMM_N, STRIDE = 16, 32, 200_000, 10


@pytest.fixture(scope="module")
def gmm_bench():
    K, d, N_ = GMM_K, GMM_D, GMM_N
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, 0)
    om = O.GmmModel(Y.astype(np.float64), K, np.zeros(d), 25 * np.eye(d), False, alpha=np.ones(K), df=d + 2,
                    scale0=np.eye(d))
    g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), alpha=np.ones(K), df=d + 2, mu=mus, cov=covs, pis=pis, z=z,
                 seed=1)
    g.sweep(2)
    return om, g


def test_gmm_disc_z_bit_exact_at_benchmark_shape(orc, gmm_bench):
    om, g = gmm_bench
    K, d, N_ = GMM_K, GMM_D, GMM_N
    st = g.state()
    z = torch.full((N_,), -1, dtype=torch.int32, device="cuda")
    L = N.lib()
    N.check(L.ab_gmm_prep(K, d, N.ptr(g.cov), N.ptr(g.Linv), N.ptr(g.hdet), N.stream_ptr()), "prep")
    N.check(L.ab_gmm_disc_z(N_, d, K, 0, N.ptr(g.Y), N.ptr(g.pis), N.ptr(g.mu), N.ptr(g.Linv), N.ptr(g.hdet),
                            N.ptr(z), 31, 17, 0, N.stream_ptr()), "disc_z")
    got = z.cpu().numpy()
    assert got.min() >= 0 and got.max() < K
    idx = np.arange(0, N_, STRIDE, dtype=np.int32)
    ref = O.gmm_disc_z_subset(orc, om, st["pis"], st["mu"], st["cov"], idx, 31, 17)
    np.testing.assert_array_equal(got[idx], ref)


def test_gmm_sweep_per_sweep_contract_at_benchmark_shape(orc, gmm_bench):
    om, g = gmm_bench
    N_ = GMM_N
    prev = g.state()
    it = g.iteration
    g.sweep(1)
    st = g.state()
    # the conjugate draws from the previous state's statistics (all N points)
    p, m, c, zz = prev["pis"].copy(), prev["mu"].copy(), prev["cov"].copy(), prev["z"].copy()
    cnt, s, _ = O.gmm_stats(orc, om, zz, m)
    np.testing.assert_array_equal(g.cnt.cpu().numpy(), cnt)
    p = O.gmm_conj_pis(orc, om, cnt, g.seed, it)
    np.testing.assert_allclose(st["pis"], p, rtol=1e-10)
    m = O.gmm_conj_mu(orc, om, cnt, s, c, g.seed, it)
    np.testing.assert_allclose(st["mu"], m, rtol=1e-8, atol=1e-8)
    _, _, obs = O.gmm_stats(orc, om, zz, st["mu"])
    c = O.gmm_conj_cov(orc, om, cnt, obs, g.seed, it)
    np.testing.assert_allclose(st["cov"], c, rtol=1e-8, atol=1e-10)
    # z bit-exact given the device's own new parameters, on every 10th point
    idx = np.arange(3, N_, STRIDE, dtype=np.int32)
    ref = O.gmm_disc_z_subset(orc, om, st["pis"], st["mu"], st["cov"], idx, g.seed, it)
    np.testing.assert_array_equal(st["z"][idx], ref)
