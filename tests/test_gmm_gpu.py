"""GPU parity of the Gaussian-mixture path against the CPU oracle.

Contract: the Cholesky / inverse / quadratic-form arithmetic repeats the
reference's operation order in binary64, so given the same weights, means,
covariances and uniforms the assignments z equal the reference's bit for bit
(exp/log of CUDA versus the C library could differ in a last bit, which
would only matter for a uniform within 1e-16 of a boundary); the
statistics are exact counts and binary64 sums in another order (1e-12
relative); conjugate draws agree to 1e-9 relative given the same statistics.
"""
import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N
from augurv2_b200.gmm import GmmGibbs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


def hmodel(N_, K, d, seed):
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, seed)
    om = O.GmmModel(Y, K, np.zeros(d), 25 * np.eye(d), False, alpha=np.ones(K), df=d + 2, scale0=np.eye(d))
    return Y, z, mus, covs, pis, om


@pytest.mark.parametrize("N_,K,d", [(3000, 16, 32), (2000, 4, 5), (500, 3, 2), (400, 5, 40)])
def test_disc_z_bit_exact(orc, N_, K, d):
    Y, z, mus, covs, pis, om = hmodel(N_, K, d, 1 + d)
    g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), alpha=np.ones(K), df=d + 2, mu=mus, cov=covs, pis=pis, seed=4)
    L = N.lib()
    N.check(L.ab_gmm_prep(K, d, N.ptr(g.cov), N.ptr(g.Linv), N.ptr(g.hdet), N.stream_ptr()), "prep")
    N.check(L.ab_gmm_disc_z(N_, d, K, 0, N.ptr(g.Y), N.ptr(g.pis), N.ptr(g.mu), N.ptr(g.Linv), N.ptr(g.hdet),
                            N.ptr(g.z), 4, 6, 0, N.stream_ptr()), "disc_z")
    got = g.z.cpu().numpy()
    ref = O.gmm_disc_z(orc, om, pis, mus, covs, 4, 6)
    np.testing.assert_array_equal(got, ref)


def test_stats_and_conj_draws(orc):
    N_, K, d = 2500, 6, 8
    Y, z, mus, covs, pis, om = hmodel(N_, K, d, 3)
    g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), alpha=np.ones(K), df=d + 2, mu=mus, cov=covs, pis=pis, z=z, seed=9)
    L = N.lib()
    st = N.stream_ptr()
    N.check(L.ab_gmm_stats(N_, d, K, N.ptr(g.Y), N.ptr(g.z), N.ptr(g.mu), N.ptr(g.cnt), N.ptr(g.sum), N.ptr(g.obs),
                           N.ptr(g.scratch), st), "stats")
    cnt, s, obs = O.gmm_stats(orc, om, z, mus)
    np.testing.assert_array_equal(g.cnt.cpu().numpy(), cnt)
    np.testing.assert_allclose(g.sum.cpu().numpy(), s, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(g.obs.cpu().numpy(), obs, rtol=1e-12, atol=1e-9)
    # conjugate draws from the oracle's exact statistics
    g.cnt.copy_(torch.as_tensor(cnt)); g.sum.copy_(torch.as_tensor(s)); g.obs.copy_(torch.as_tensor(obs))
    N.check(L.ab_gmm_conj_pis(K, N.ptr(g.alpha), N.ptr(g.cnt), N.ptr(g.pis), 9, 2, 0, st), "pis")
    np.testing.assert_allclose(g.pis.cpu().numpy(), O.gmm_conj_pis(orc, om, cnt, 9, 2), rtol=1e-12)
    N.check(L.ab_gmm_conj_mu(K, d, 0, N.ptr(g.mu0), N.ptr(g.cov0), N.ptr(g.cnt), N.ptr(g.sum), N.ptr(g.cov),
                             N.ptr(g.mu), 9, 2, 0, st), "mu")
    np.testing.assert_allclose(g.mu.cpu().numpy(), O.gmm_conj_mu(orc, om, cnt, s, covs, 9, 2), rtol=1e-9, atol=1e-9)
    N.check(L.ab_gmm_conj_cov(K, d, d + 2, N.ptr(g.scale0), N.ptr(g.cnt), N.ptr(g.obs), N.ptr(g.cov), 9, 2, 0, st),
            "cov")
    np.testing.assert_allclose(g.cov.cpu().numpy(), O.gmm_conj_cov(orc, om, cnt, obs, 9, 2), rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("K,d", [(16, 32), (3, 5)])
def test_conj_cov_in_two_calls_equals_one(K, d):
    """ab_gmm_bartlett + ab_gmm_conj_cov_chi (the sweep's split, the first on
    a side stream) give ab_gmm_conj_cov's draw bit for bit."""
    rng = np.random.default_rng(K + d)
    cnt = torch.as_tensor(rng.integers(0, 5000, size=K).astype(np.int32)).cuda()
    a = rng.standard_normal((K, d, d))
    obs = torch.as_tensor(np.einsum("kij,klj->kil", a, a) * 50.0).cuda()
    scale0 = torch.eye(d, dtype=torch.float64, device="cuda")
    one = torch.zeros((K, d, d), dtype=torch.float64, device="cuda")
    two = torch.zeros_like(one)
    chi = torch.zeros((K, d), dtype=torch.float64, device="cuda")
    L = N.lib()
    st = N.stream_ptr()
    N.check(L.ab_gmm_conj_cov(K, d, d + 2, N.ptr(scale0), N.ptr(cnt), N.ptr(obs), N.ptr(one), 5, 3, 0, st), "cov")
    N.check(L.ab_gmm_bartlett(K, d, d + 2, N.ptr(cnt), N.ptr(chi), 5, 3, 0, st), "bartlett")
    N.check(L.ab_gmm_conj_cov_chi(K, d, d + 2, N.ptr(scale0), N.ptr(cnt), N.ptr(obs), N.ptr(chi), N.ptr(two), 5, 3,
                                  0, st), "cov_chi")
    torch.cuda.synchronize()
    assert torch.equal(one, two)
    assert torch.isfinite(one).all()


@pytest.mark.parametrize("N_,K,d", [(300_000, 16, 32), (250_000, 3, 40), (1, 2, 3), (900, 16, 2)])
def test_stats_sizes(orc, N_, K, d):
    """Statistics at sizes where a CTA's chunk spans several shared-memory
    sub-chunks (N = 3e5 at d = 32), the widest d of the pass, a single point,
    and many components with few points each; a label outside [0, K) is not
    counted."""
    rng = np.random.default_rng(N_ + d)
    Y = rng.standard_normal((N_, d)).astype(np.float32) * 3
    z = rng.integers(0, K, size=N_).astype(np.int32)
    mus = rng.standard_normal((K, d))
    om = O.GmmModel(Y.astype(np.float64), K, np.zeros(d), 25 * np.eye(d), False, alpha=np.ones(K), df=d + 2,
                    scale0=np.eye(d))
    g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), alpha=np.ones(K), df=d + 2, mu=mus, z=z, seed=1)
    if N_ > 10:
        g.z[N_ // 2] = K + 3                     # not a component: skipped
    L = N.lib()
    N.check(L.ab_gmm_stats(N_, d, K, N.ptr(g.Y), N.ptr(g.z), N.ptr(g.mu), N.ptr(g.cnt), N.ptr(g.sum), N.ptr(g.obs),
                           N.ptr(g.scratch), N.stream_ptr()), "stats")
    keep = np.ones(N_, bool)
    if N_ > 10:
        keep[N_ // 2] = False
    cnt = np.bincount(z[keep], minlength=K)
    s = np.zeros((K, d))
    obs = np.zeros((K, d, d))
    Y64 = Y.astype(np.float64)
    for k in range(K):
        m = keep & (z == k)
        s[k] = Y64[m].sum(0)
        c = Y64[m] - mus[k]
        obs[k] = c.T @ c
    np.testing.assert_array_equal(g.cnt.cpu().numpy(), cnt)
    np.testing.assert_allclose(g.sum.cpu().numpy(), s, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(g.obs.cpu().numpy(), obs, rtol=1e-12, atol=1e-8)


def test_hmvgmm_sweeps_per_sweep_contract(orc):
    N_, K, d = 1500, 4, 5
    Y, z, mus, covs, pis, om = hmodel(N_, K, d, 11)
    g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), alpha=np.ones(K), df=d + 2, mu=mus, cov=covs, pis=pis, z=z,
                 seed=3)
    for it in range(4):
        prev = g.state()
        g.sweep(1)
        st = g.state()
        # the oracle sweep from the GPU's previous state
        p, m, c, zz = prev["pis"].copy(), prev["mu"].copy(), prev["cov"].copy(), prev["z"].copy()
        O.gmm_sweep(orc, om, p, m, c, zz, 3, it)
        np.testing.assert_allclose(st["pis"], p, rtol=1e-10)
        np.testing.assert_allclose(st["mu"], m, rtol=1e-8, atol=1e-8)
        np.testing.assert_allclose(st["cov"], c, rtol=1e-8, atol=1e-10)
        # z bit-exact given the GPU's own new parameters
        z_ref = O.gmm_disc_z(orc, om, st["pis"], st["mu"], st["cov"], 3, it)
        np.testing.assert_array_equal(st["z"], z_ref)


@pytest.mark.parametrize("move", ["conj", "eslice", "mwg"])
def test_mvgmm_moves(orc, move):
    rng = np.random.default_rng(5)
    K, d, N_ = 3, 2, 300
    centres = np.array([[0.0, 2.0], [2.0, -2.0], [-2.0, -2.0]])
    covs = 0.1 * np.eye(d)
    Y = (centres[np.arange(N_) % K] + rng.standard_normal((N_, d)) * np.sqrt(0.1)).astype(np.float32).astype(np.float64)
    pis = np.full(K, 1.0 / K)
    om = O.GmmModel(Y, K, np.zeros(d), np.eye(d), True)
    mu0 = centres + 0.3 * rng.standard_normal((K, d))
    z0 = (np.arange(N_) % K).astype(np.int32)
    g = GmmGibbs(Y, K, np.zeros(d), np.eye(d), pis=pis, covs=covs, mu=mu0, z=z0, move=move,
                 prop_cov=0.05 * np.eye(d), seed=2)
    for it in range(3):
        prev = g.state()
        g.sweep(1)
        st = g.state()
        if move == "conj":
            m = prev["mu"].copy()
            cnt, s, _ = O.gmm_stats(orc, om, prev["z"], m)
            m = O.gmm_conj_mu(orc, om, cnt, s, covs, 2, it)
        elif move == "eslice":
            m = O.gmm_eslice(orc, om, prev["mu"], covs, prev["z"], 2, it)
        else:
            m = O.gmm_mwg(orc, om, prev["mu"], covs, prev["z"], 0.05 * np.eye(d), 2, it)
        np.testing.assert_allclose(st["mu"], m, rtol=1e-9, atol=1e-9)
        np.testing.assert_array_equal(st["z"], O.gmm_disc_z(orc, om, pis, st["mu"], covs, 2, it))


def test_bench_shape_properties():
    """K=16, d=32, N=2e5 (the benchmark shape): statistics sum to N, the
    covariances stay symmetric positive definite, assignments recover most
    of the generating components' structure."""
    K, d, N_ = 16, 32, 200000
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, 0)
    g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), alpha=np.ones(K), df=d + 2, mu=mus, cov=covs, pis=pis, z=z,
                 seed=1)
    g.sweep(3)
    st = g.state()
    assert int(g.cnt.sum()) == N_
    for k in range(K):
        c = st["cov"][k]
        np.testing.assert_allclose(c, c.T, rtol=0, atol=1e-12)
        assert np.linalg.eigvalsh(c).min() > 0
    assert abs(st["pis"].sum() - 1) < 1e-12
