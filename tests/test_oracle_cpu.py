"""Pins the CPU oracle: Philox known-answer vectors, the golden fixtures made
from the reference's own runtime, and (when the reference build is present)
live bit-for-bit agreement with it."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


@pytest.fixture(scope="module")
def ref():
    if not O.available("ref"):
        pytest.skip("reference build oracle/_ref not present")
    return O.Oracle("ref")


# Random123 known-answer vectors for philox4x32-10.
KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
]


@pytest.mark.parametrize("ctr,key,expect", KAT)
def test_philox_kat(orc, ctr, key, expect):
    assert list(orc.philox_block(ctr, key)) == expect


def test_uniforms_open_interval(orc):
    u = orc.draws(1, 2, 3, 4, 20000)
    assert u.min() > 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.01
    n = orc.draws(1, 2, 3, 5, 20000, normal=True)
    assert abs(n.mean()) < 0.03 and abs(n.std() - 1.0) < 0.03


def test_primitives_golden(orc):
    g = np.load(os.path.join(GOLD, "primitives.npz"))
    shapes = list(g["shapes"]) + [2.0, 0.3]
    rates = [1.0] * len(g["shapes"]) + [0.5, 4.0]
    got = np.array([[orc.gamma_sample(s, r, 11, e, 3, O.TAG_PHI) for e in range(8)]
                    for s, r in zip(shapes, rates)])
    np.testing.assert_array_equal(got, g["gamma"])
    disc = [orc.unnorm_disc_samp(p, 19, i, 2, O.TAG_Z) for i, p in enumerate(g["pmfs"])]
    np.testing.assert_array_equal(disc, g["disc"])


def test_lda_golden_reference_fixture(orc):
    """examples/lda.py d4_k4_v8 corpus: 10 sweeps equal the reference's."""
    g = np.load(os.path.join(GOLD, "lda_d4_k4_v8.npz"))
    D, K, V = 4, 4, 8
    theta, phi = np.full((D, K), 1.0 / K), np.full((K, V), 1.0 / V)
    z = np.zeros(len(g["w"]), np.int32)
    for s in range(10):
        orc.lda_sweeps(g["doc_off"], g["w"], g["alpha"], g["beta"], theta, phi, z, 0, s, 1)
        np.testing.assert_array_equal(theta, g["theta"][s])
        np.testing.assert_array_equal(phi, g["phi"][s])
        np.testing.assert_array_equal(z, g["z"][s])


def test_lda_golden_synthetic(orc):
    g = np.load(os.path.join(GOLD, "lda_k12_v300_d40.npz"))
    th, ph, z = g["theta0"].copy(), g["phi0"].copy(), g["z0"].copy()
    orc.lda_sweeps(g["doc_off"], g["w"], g["alpha"], g["beta"], th, ph, z, 7, 0, 3)
    np.testing.assert_array_equal(th, g["theta"])
    np.testing.assert_array_equal(ph, g["phi"])
    np.testing.assert_array_equal(z, g["z"])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_lda_oracle_vs_reference_live(orc, ref, seed):
    rng = np.random.default_rng(seed)
    D, K, V = 7, 5, 23
    lens = rng.integers(0, 15, size=D)          # includes empty documents
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    w = rng.integers(0, V, size=off[-1]).astype(np.int32)
    alpha, beta = rng.random(K) + 0.05, rng.random(V) * 0.1 + 0.005
    th0 = rng.dirichlet(np.ones(K), size=D); ph0 = rng.dirichlet(np.ones(V), size=K)
    z0 = rng.integers(0, K, size=off[-1]).astype(np.int32)
    a = orc.lda_sweeps(off, w, alpha, beta, th0.copy(), ph0.copy(), z0.copy(), seed, 5, 4)
    b = ref.lda_sweeps(off, w, alpha, beta, th0.copy(), ph0.copy(), z0.copy(), seed, 5, 4)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_gamma_oracle_vs_reference_live(orc, ref):
    for s in [0.001, 0.02, 0.7, 1.0, 1.5, 8.0, 1e3]:
        for e in range(50):
            assert orc.gamma_sample(s, 1.3, 3, e, 1, 2) == ref.gamma_sample(s, 1.3, 3, e, 1, 2)


def test_gamma_moments(orc):
    for s in [0.1, 1.0, 4.0]:
        x = np.array([orc.gamma_sample(s, 2.0, 9, e, 0, 2) for e in range(20000)])
        assert abs(x.mean() - s / 2.0) < 5 * np.sqrt(s / 4.0 / 20000)


# ---- HLR ------------------------------------------------------------------
def _hlr_model(g, compat=True):
    vprior = "exponential" if int(g["vprior"]) == 0 else "invgamma"
    return O.HlrModel(g["X"], g["y"], has_b=bool(g["has_b"]), vprior=vprior, lam=1.0, a0=1.0,
                      s0=1.0, compat=compat)


@pytest.mark.parametrize("name", ["hlr", "ighlr"])
def test_hlr_golden_ll_grad(orc, name):
    g = np.load(os.path.join(GOLD, name + "_golden.npz"))
    m = _hlr_model(g)
    for key in [k for k in g.files if k.startswith("ll_")]:
        b = key[3:]
        idx = g["idx_" + b]
        ll = np.array([O.hlr_ll(orc, m, p, idx) for p in g["pars"]])
        gr = np.array([O.hlr_grad(orc, m, p, idx) for p in g["pars"]])
        np.testing.assert_array_equal(ll, g[key])
        np.testing.assert_array_equal(gr, g["grad_" + b])


@pytest.mark.parametrize("name", ["hlr", "ighlr"])
def test_hlr_golden_transitions(orc, name):
    g = np.load(os.path.join(GOLD, name + "_golden.npz"))
    m = _hlr_model(g)
    D = int(g["D"])
    p = g["par0"].copy()
    for it in range(6):
        O.hlr_hmc(orc, m, p, g["idx_theta"], 0.3, 0.05, 7, it)
        np.testing.assert_array_equal(p, g["hmc"][it])
    p = g["par0"].copy()
    for it in range(6):
        O.hlr_nuts(orc, m, p, g["idx_joint"], 0.05, 7, it)
        np.testing.assert_array_equal(p, g["nuts"][it])
    p = g["par0"].copy()
    for it in range(6):
        O.hlr_mwg(orc, m, p, D + 1, 0.5, 7, it)
        np.testing.assert_array_equal(p, g["mwg"][it])
    p = g["par0"].copy()
    for it in range(8):
        O.hlr_rslice(orc, m, p, g["idx_theta"], 0.5, 0.05, 7, it)
        np.testing.assert_array_equal(p, g["rslice"][it])


@pytest.mark.parametrize("seed", [0, 1])
def test_hlr_oracle_vs_reference_live(orc, ref, seed):
    X, y, beta, s2 = O.hlr_synthetic(90, 3, seed, has_b=True)
    m = O.HlrModel(X, y, has_b=True, vprior="exponential")
    D = 3
    par = np.concatenate([beta, [0.1], [1.0]])
    for idx in [[0, 1, 2], [3], [4], [4, 3, 0, 1, 2]]:
        assert O.hlr_ll(orc, m, par, idx) == O.hlr_ll(ref, m, par, idx)
        np.testing.assert_array_equal(O.hlr_grad(orc, m, par, idx), O.hlr_grad(ref, m, par, idx))
    for it in range(4):
        a, b = par.copy(), par.copy()
        O.hlr_nuts(orc, m, a, [4, 3, 0, 1, 2], 0.1, seed, it)
        O.hlr_nuts(ref, m, b, [4, 3, 0, 1, 2], 0.1, seed, it)
        np.testing.assert_array_equal(a, b)
    a, b = par.copy(), par.copy()
    refl = 0
    for it in range(10):
        _, _, r = O.hlr_rslice(orc, m, a, [0, 1, 2, 3], 1.0, 0.08, seed, it, chain=2, comp=1)
        O.hlr_rslice(ref, m, b, [0, 1, 2, 3], 1.0, 0.08, seed, it, chain=2, comp=1)
        np.testing.assert_array_equal(a, b)
        refl += r
    assert refl > 0, "the chain never left the slice: reflections untested"


def test_hlr_gradient_finite_difference(orc):
    """Exact-density gradient against central differences (the idea of
    h_augur_chk_grad, cbits/augur_mcmclib.h:199-250)."""
    X, y, beta, s2 = O.hlr_synthetic(300, 4, 5, has_b=True)
    m = O.HlrModel(X, y, has_b=True, vprior="exponential", compat=False)
    par = np.concatenate([beta * 0.3, [0.2], [0.8]])
    idx = [5, 4, 0, 1, 2, 3]
    g = O.hlr_grad(orc, m, par, idx)
    h = 1e-6
    for j, i in enumerate(idx):
        pp, pm = par.copy(), par.copy()
        pp[i] += h; pm[i] -= h
        fd = (O.hlr_ll(orc, m, pp, idx) - O.hlr_ll(orc, m, pm, idx)) / (2 * h)
        assert abs(fd - g[j]) <= 1e-5 * max(1.0, abs(g[j]))


def _glm_data(lik, N, D, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((N, D))
    beta = rng.standard_normal(D) * 0.3
    t = X @ beta + 0.1
    if lik == "poisson":
        y = rng.poisson(np.exp(t)).astype(np.int32)
    else:
        y = t + rng.standard_normal(N) * 0.7
    return X, y, beta


@pytest.mark.parametrize("lik", ["poisson", "normal"])
def test_glm_oracle_vs_reference_live(orc, ref, lik):
    """Poisson(exp(t)) and Normal(t, obs_var) likelihoods with the HLR priors:
    the oracle's restatement equals the reference's own cbits densities,
    adjoints and NUTS / HMC transitions bit for bit."""
    X, y, beta = _glm_data(lik, 80, 3, 11)
    m = O.HlrModel(X, y, has_b=True, vprior="invgamma", lik=lik, obs_var=0.49)
    par = np.concatenate([beta, [0.1], [1.3]])
    for idx in [[0, 1, 2], [3], [4], [4, 3, 0, 1, 2]]:
        assert O.hlr_ll(orc, m, par, idx) == O.hlr_ll(ref, m, par, idx)
        np.testing.assert_array_equal(O.hlr_grad(orc, m, par, idx), O.hlr_grad(ref, m, par, idx))
    for it in range(4):
        a, b = par.copy(), par.copy()
        O.hlr_nuts(orc, m, a, [4, 3, 0, 1, 2], 0.05, 3, it)
        O.hlr_nuts(ref, m, b, [4, 3, 0, 1, 2], 0.05, 3, it)
        np.testing.assert_array_equal(a, b)
        a, b = par.copy(), par.copy()
        O.hlr_hmc(orc, m, a, [0, 1, 2, 3], 0.2, 0.04, 3, it)
        O.hlr_hmc(ref, m, b, [0, 1, 2, 3], 0.2, 0.04, 3, it)
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("lik", ["poisson", "normal"])
def test_glm_gradient_finite_difference(orc, lik):
    X, y, beta = _glm_data(lik, 200, 4, 12)
    m = O.HlrModel(X, y, has_b=True, vprior="exponential", compat=False, lik=lik, obs_var=0.5)
    par = np.concatenate([beta * 0.5, [0.2], [0.8]])
    idx = [5, 4, 0, 1, 2, 3]
    g = O.hlr_grad(orc, m, par, idx)
    h = 1e-6
    for j, i in enumerate(idx):
        pp, pm = par.copy(), par.copy()
        pp[i] += h; pm[i] -= h
        fd = (O.hlr_ll(orc, m, pp, idx) - O.hlr_ll(orc, m, pm, idx)) / (2 * h)
        assert abs(fd - g[j]) <= 1e-5 * max(1.0, abs(g[j]))


# ---- Gaussian mixtures ---------------------------------------------------------
def test_mvgmm_golden_reference_example(orc):
    g = np.load(os.path.join(GOLD, "mvgmm_k3_d2.npz"))
    K, d = g["mu"].shape[1:]
    m = O.GmmModel(g["Y"], K, g["mu0"], g["cov0"], True)
    mu, z = np.zeros((K, d)), np.zeros(len(g["Y"]), np.int32)
    pis = g["pis"].copy()
    for it in range(8):
        O.gmm_sweep(orc, m, pis, mu, g["covs"].copy(), z, 1, it)
        np.testing.assert_array_equal(mu, g["mu"][it])
        np.testing.assert_array_equal(z, g["z"][it])
    np.testing.assert_array_equal(O.gmm_eslice(orc, m, g["mu"][-1], g["covs"], g["z"][-1], 2, 0), g["eslice"])
    np.testing.assert_array_equal(O.gmm_mwg(orc, m, g["mu"][-1], g["covs"], g["z"][-1], g["cov0"], 2, 0), g["mwg"])


def test_hmvgmm_golden(orc):
    g = np.load(os.path.join(GOLD, "hmvgmm_k4_d5.npz"))
    K, d = g["mu_init"].shape
    m = O.GmmModel(g["Y"], K, np.zeros(d), 25 * np.eye(d), False, alpha=np.ones(K), df=d + 2, scale0=np.eye(d))
    pis, mu, cov, z = (g["pis_init"].copy(), g["mu_init"].copy(), g["cov_init"].copy(), g["z_init"].copy())
    for it in range(4):
        O.gmm_sweep(orc, m, pis, mu, cov, z, 3, it)
        np.testing.assert_array_equal(pis, g["pis"][it])
        np.testing.assert_array_equal(mu, g["mu"][it])
        np.testing.assert_array_equal(cov, g["cov"][it])
        np.testing.assert_array_equal(z, g["z"][it])


def test_gmm_oracle_vs_reference_live(orc, ref):
    Y, z, mus, covs, pis = O.gmm_synthetic(150, 3, 4, seed=9)
    m = O.GmmModel(Y, 3, np.zeros(4), 9 * np.eye(4), False, alpha=np.full(3, 2.0), df=7, scale0=2 * np.eye(4))
    np.testing.assert_array_equal(O.gmm_disc_z(orc, m, pis, mus, covs, 8, 2),
                                  O.gmm_disc_z(ref, m, pis, mus, covs, 8, 2))
    for a, b in zip(O.gmm_stats(orc, m, z, mus), O.gmm_stats(ref, m, z, mus)):
        np.testing.assert_array_equal(a, b)
    cnt, s, obs = O.gmm_stats(orc, m, z, mus)
    np.testing.assert_array_equal(O.gmm_conj_mu(orc, m, cnt, s, covs, 8, 2), O.gmm_conj_mu(ref, m, cnt, s, covs, 8, 2))
    np.testing.assert_array_equal(O.gmm_conj_cov(orc, m, cnt, obs, 8, 2), O.gmm_conj_cov(ref, m, cnt, obs, 8, 2))
    np.testing.assert_array_equal(O.gmm_eslice(orc, m, mus, covs, z, 8, 2), O.gmm_eslice(ref, m, mus, covs, z, 8, 2))


def test_gmm_disc_z_subset_equals_full_pass(orc):
    """The subset draw gives each listed point the value of the full pass
    (same substream per point), in the order listed."""
    Y, z, mus, covs, pis = O.gmm_synthetic(400, 5, 6, seed=4)
    m = O.GmmModel(Y, 5, np.zeros(6), 9 * np.eye(6), False, alpha=np.ones(5), df=8, scale0=np.eye(6))
    full = O.gmm_disc_z(orc, m, pis, mus, covs, 6, 3)
    idx = np.array([399, 0, 7, 7, 123, 250], np.int32)
    np.testing.assert_array_equal(O.gmm_disc_z_subset(orc, m, pis, mus, covs, idx, 6, 3), full[idx])


def test_mvnormal_ll_matches_scipy(orc):
    from scipy.stats import multivariate_normal
    rng = np.random.default_rng(0)
    A = rng.standard_normal((6, 6))
    cov = A @ A.T + 6 * np.eye(6)
    x, mu = rng.standard_normal(6), rng.standard_normal(6)
    assert abs(O.mvnormal_ll(orc, x, mu, cov) - multivariate_normal(mu, cov).logpdf(x)) < 1e-10


def _conj_cases():
    import sys
    sys.path.insert(0, GOLD)
    import make_golden as M
    return M


@pytest.mark.parametrize("kind", range(7))
def test_conj_scalar_golden(orc, kind):
    """The scalar conjugate restatement against fixtures from the reference's
    own samplers (augur_dist.c:185-195, 314-336, 408-412), bit for bit."""
    M = _conj_cases()
    g = np.load(os.path.join(GOLD, "conj_scalar.npz"))
    name = M.CONJ_KINDS[kind]
    off, x, aux, h0, h1, h2 = M.conj_inputs(name, 100 + kind)
    for it in (0, 5):
        out, ssum, saux = orc.conj_scalar(kind, off, x, h0, h1, h2, aux=aux, seed=23, it=it)
        np.testing.assert_array_equal(out, g["%s_it%d_out" % (name, it)])
        np.testing.assert_array_equal(ssum, g["%s_it%d_sum" % (name, it)])
        np.testing.assert_array_equal(saux, g["%s_it%d_aux" % (name, it)])


@pytest.mark.parametrize("kind", range(7))
def test_conj_scalar_live(orc, ref, kind):
    M = _conj_cases()
    off, x, aux, h0, h1, h2 = M.conj_inputs(M.CONJ_KINDS[kind], 300 + kind)
    for seed, it in ((1, 0), (99, 12)):
        a = orc.conj_scalar(kind, off, x, h0, h1, h2, aux=aux, seed=seed, it=it)
        b = ref.conj_scalar(kind, off, x, h0, h1, h2, aux=aux, seed=seed, it=it)
        for u, v in zip(a, b):
            np.testing.assert_array_equal(u, v)


def test_ll_mod_oracle_vs_reference_live(orc, ref):
    """The model log density (augur_get_curr_ll's ll_mod) of the restatement
    equals the reference runtime's, LDA and both mixture models."""
    from augurv2_b200.lda import synthetic_corpus
    K, V, D = 5, 40, 12
    off, w = synthetic_corpus(K, V, D, 20, 0.3, 0.1, seed=2)
    rng = np.random.default_rng(2)
    theta = rng.dirichlet(np.full(K, 0.5), size=D)
    phi = rng.dirichlet(np.full(V, 0.2), size=K)
    z = rng.integers(0, K, size=len(w)).astype(np.int32)
    alpha, beta = np.full(K, 0.3), np.full(V, 0.1)
    a = orc.lda_ll_mod(off, w, z, alpha, beta, theta, phi)
    assert a == ref.lda_ll_mod(off, w, z, alpha, beta, theta, phi)
    doc = np.repeat(np.arange(D), np.diff(off))
    expect = ((alpha - 1) * np.log(theta)).sum() + ((beta - 1) * np.log(phi)).sum() + \
        np.log(theta[doc, z]).sum() + np.log(phi[z, w]).sum()
    assert abs(a - expect) <= 1e-10 * abs(expect)
    Y, zg, mus, covs, pis = O.gmm_synthetic(200, 3, 4, seed=5)
    for shared in (False, True):
        m = O.GmmModel(Y, 3, np.zeros(4), 9 * np.eye(4), shared, alpha=np.full(3, 2.0), df=7,
                       scale0=2 * np.eye(4))
        cv = covs[0] if shared else covs
        assert O.gmm_ll_mod(orc, m, pis, mus, cv, zg) == O.gmm_ll_mod(ref, m, pis, mus, cv, zg)


def test_invwishart_ll_against_scipy(orc):
    """The reference's inverse-Wishart log density equals scipy's up to its
    log(3.1415) in the multivariate gamma (augur_math.c:80-86)."""
    from scipy.stats import invwishart
    from scipy.special import multigammaln
    d, df = 4, 7
    Y, zg, mus, covs, pis = O.gmm_synthetic(10, 1, d, seed=1)
    m = O.GmmModel(Y, 1, np.zeros(d), np.eye(d), False, alpha=np.ones(1), df=df, scale0=2 * np.eye(d))
    got = O.gmm_ll_mod(orc, m, np.ones(1), np.zeros((1, d)), covs, np.zeros(10, np.int32))
    rest = O.mvnormal_ll(orc, np.zeros(d), np.zeros(d), np.eye(d)) + sum(
        O.mvnormal_ll(orc, Y[n], np.zeros(d), covs[0]) for n in range(10))
    quirk = d * (d - 1) / 4 * (np.log(np.pi) - np.log(3.1415))
    expect = invwishart(df=df, scale=2 * np.eye(d)).logpdf(covs[0]) + quirk
    np.testing.assert_allclose(got - rest, expect, rtol=1e-10)
    assert abs(multigammaln(3.5, d) - (d * (d - 1) / 4 * np.log(np.pi) + sum(
        __import__("math").lgamma(3.5 - i / 2) for i in range(d)))) < 1e-10


def test_predictive_ll_against_scipy(orc):
    """Held-out log-likelihoods (experiments/lda/lda.py:149-173,
    experiments/hmvgmm/hmvgmm.py:143-178) against scipy's logsumexp and
    multivariate normal."""
    from scipy.special import logsumexp
    from scipy.stats import multivariate_normal as mvn
    rng = np.random.default_rng(7)
    K, V, D = 6, 30, 9
    off = np.concatenate([[0], np.cumsum(rng.integers(0, 8, size=D))]).astype(np.int32)
    w = rng.integers(0, V, size=off[-1]).astype(np.int32)
    theta = rng.dirichlet(np.full(K, 0.5), size=D)
    phi = rng.dirichlet(np.full(V, 0.3), size=K)
    doc = np.repeat(np.arange(D), np.diff(off))
    expect = logsumexp(np.log(theta[doc]) + np.log(phi[:, w].T), axis=1).sum()
    np.testing.assert_allclose(orc.lda_pred_ll(off, w, theta, phi), expect, rtol=1e-12)
    Y, zg, mus, covs, pis = O.gmm_synthetic(150, 4, 3, seed=3)
    lp = np.stack([mvn(mus[k], covs[k]).logpdf(Y) + np.log(pis[k]) for k in range(4)], 1)
    np.testing.assert_allclose(O.gmm_pred_ll(orc, Y, pis, mus, covs), logsumexp(lp, axis=1).sum(), rtol=1e-10)
    lp = np.stack([mvn(mus[k], covs[0]).logpdf(Y) + np.log(pis[k]) for k in range(4)], 1)
    np.testing.assert_allclose(O.gmm_pred_ll(orc, Y, pis, mus, covs[0], shared_cov=True),
                               logsumexp(lp, axis=1).sum(), rtol=1e-10)
