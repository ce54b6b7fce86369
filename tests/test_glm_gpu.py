"""The per-chain HLR engine with the other generalised-linear likelihoods the
reference's modelling language can state on t = dotprod(theta, x[n]) + b:
y[n] ~ Poisson(exp(t)) and y[n] ~ Normal(t, s2), priors as hlr.rv.

Parity against the FP64 oracle, itself equal to the reference's cbits
densities and adjoints (tests/test_oracle_cpu.py, test_glm_oracle_vs_reference_live).
Tolerances as tests/test_hlr_gpu.py: the data terms run in FP32 with
compensated sums, so block log densities agree within 1e-5 relative to the
sum of the terms' magnitudes and each gradient component within 1e-5 of
sum_n |r_n x_nk| plus the prior term; HMC transitions from the same state and
substreams agree to 1e-4 when the accept decision agrees."""
import math

import numpy as np
import pytest
import torch

from augurv2_b200 import hlr as H
from augurv2_b200.augurdistlib import AugurDefault
from augurv2_b200.augurlib import AugurInfer, AugurOpt
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


def glm_data(lik, N, D, seed, obs_var=0.5):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((N, D))
    beta = rng.standard_normal(D) * (0.3 / np.sqrt(max(D / 8, 1)))
    t = X @ beta + 0.2
    if lik == "poisson":
        y = rng.poisson(np.exp(t)).astype(np.int32)
    else:
        y = t + rng.standard_normal(N) * np.sqrt(obs_var)
    return X, y, beta


def _models(lik, X, y, has_b, vprior, compat, obs_var=0.5):
    om = O.HlrModel(X, y, has_b=has_b, vprior=vprior, compat=compat, lik=lik, obs_var=obs_var)
    gd = H.HlrData(X, y, has_b=has_b, vprior=vprior, compat=compat, lik=lik, obs_var=obs_var)
    return om, gd


def _residual(lik, y, t, obs_var):
    return np.abs(y - np.exp(t)) if lik == "poisson" else np.abs(y - t) / obs_var


@pytest.mark.parametrize("lik", ["poisson", "normal"])
@pytest.mark.parametrize("N,D,has_b,vprior,compat", [(2000, 8, True, "exponential", True),
                                                     (1500, 40, False, "invgamma", False),
                                                     (700, 13, True, "invgamma", True)])
def test_glm_ll_grad_matches_fp64_oracle(orc, lik, N, D, has_b, vprior, compat):
    X, y, beta = glm_data(lik, N, D, N + D)
    om, gd = _models(lik, X, y, has_b, vprior, compat)
    rng = np.random.default_rng(2)
    C = 5
    pars = np.zeros((C, D + 2))
    pars[:, :D] = beta + 0.1 * rng.standard_normal((C, D))
    pars[:, D] = 0.2 + 0.05 * rng.standard_normal(C) if has_b else 0.0
    pars[:, D + 1] = 0.5 + rng.random(C)
    blocks = [list(range(D)), [D + 1], [D + 1] + ([D] if has_b else []) + list(range(D))]
    if has_b:
        blocks.append([D])
    for idx in blocks:
        ll, g = H.ll_grad(gd, pars, idx)
        for c in range(C):
            l_ref = O.hlr_ll(orc, om, pars[c], idx)
            g_ref = O.hlr_grad(orc, om, pars[c], idx)
            t = X @ pars[c, :D] + (pars[c, D] if has_b else 0.0)
            if lik == "poisson":
                terms = np.abs(y * t) + np.exp(t) + np.abs([math.lgamma(k + 1.0) for k in y])
            else:
                terms = 0.5 * (y - t) ** 2 / 0.5 + abs(np.log(0.5))
            assert abs(ll[c] - l_ref) <= 1e-5 * (terms.sum() + abs(l_ref)) + 1e-9, (idx[:3], c, ll[c], l_ref)
            r = _residual(lik, y, t, 0.5)
            scale_th = np.abs(X).T @ r + np.abs(pars[c, :D]) / pars[c, D + 1]
            for j, i in enumerate(idx):
                if i < D:
                    tol = 1e-5 * scale_th[i] + 1e-9
                elif i == D:
                    tol = 1e-5 * (r.sum() + abs(pars[c, D]) / pars[c, D + 1]) + 1e-9
                else:
                    tol = 1e-9 * max(1.0, abs(g_ref[j]))
                assert abs(g[c, j] - g_ref[j]) <= tol, (idx[:3], c, j, g[c, j], g_ref[j])


@pytest.mark.parametrize("lik", ["poisson", "normal"])
def test_glm_hmc_and_nuts_transitions_match_oracle(orc, lik):
    D = 6
    X, y, beta = glm_data(lik, 800, D, 9)
    om, gd = _models(lik, X, y, True, "exponential", True)
    block = ["v", "b", "theta"]
    idx = H.block_indices(block, D)
    par0 = np.concatenate([beta, [0.2], [0.7]])
    agree, par = 0, par0.copy()
    for it in range(8):
        p_ref = par.copy()
        acc, L, prop = O.hlr_hmc(orc, om, p_ref, idx, 0.05, 0.005, 5, it)
        ch = H.HlrChains(gd, [{"kind": "HMC", "block": block, "simlen": 0.05, "eps": 0.005}], C=1, init=par,
                         seed=5, iter0=it)
        ch.run(1)
        if int(ch.stats.cpu().numpy()[0, 0, 0]) == acc:
            agree += 1
            np.testing.assert_allclose(ch.state()[0], p_ref, rtol=1e-4, atol=1e-6)
        par = p_ref
    assert agree >= 7
    # NUTS: the same tree depths and end points as the oracle's walk
    par = par0.copy()
    for it in range(4):
        p_ref = par.copy()
        depth, leaves, ovf = O.hlr_nuts(orc, om, p_ref, idx, 0.004, 6, it, max_depth=6)
        ch = H.HlrChains(gd, [{"kind": "NUTS", "block": block, "eps": 0.004, "max_depth": 6}], C=1, init=par,
                         seed=6, iter0=it)
        ch.run(1)
        st = ch.stats.cpu().numpy()
        assert int(st[0, 0, 1]) == depth
        np.testing.assert_allclose(ch.state()[0], p_ref, rtol=1e-4, atol=1e-6)
        par = p_ref


POISSON_RV = """(K : Int, N : Int, lam : Real, x : Vec (Vec Real)) => {
  param v ~ Exponential(lam) ;
  param b ~ Normal(0.0, v) ;
  param theta[k] ~ Normal(0.0, v)
      for k <- 0 until K ;
  data y[n] ~ Poisson( exp(dotprod(theta, x[n]) + b) )
      for n <- 0 until N ;
}"""

NORMAL_RV = """(K : Int, N : Int, a0 : Real, s0 : Real, s2 : Real, x : Vec (Vec Real)) => {
  param v ~ InvGamma(a0, s0) ;
  param theta[k] ~ Normal(0.0, v)
      for k <- 0 until K ;
  data y[n] ~ Normal(dotprod(theta, x[n]), s2)
      for n <- 0 until N ;
}"""


@pytest.mark.parametrize("kind", ["poisson", "normal"])
def test_glm_models_through_augur_infer(kind):
    """A Poisson and a linear regression written in the reference's modelling
    language run through AugurInfer on the device and recover their
    coefficients (posterior means within a few posterior sds of the truth)."""
    D, N = 4, 3000
    rng = np.random.default_rng(31)
    X = rng.standard_normal((N, D))
    beta = np.array([0.4, -0.3, 0.2, 0.1])
    if kind == "poisson":
        y = rng.poisson(np.exp(X @ beta + 0.3)).astype(np.int32)
        src, sched = POISSON_RV, "NUTS [v, b, theta] [0.02]"
        hyp = (D, N, 1.0, X)
    else:
        y = X @ beta + rng.standard_normal(N) * 0.5
        src, sched = NORMAL_RV, "HMC [theta] [0.2, 0.01] (*) MWG [v] ~ Normal(v, 0.3)"
        hyp = (D, N, 1.0, 1.0, 0.25, X)
    with AugurInfer("config.yml", src) as infer:
        infer.set_compile_opt(AugurOpt(cached=False, target="cpu", initStrat=AugurDefault(), seed=2))
        infer.set_user_sched(sched)
        infer.compile(*hyp)(y)
        samples = infer.samplen(burnIn=200, numSamples=400)
    th = np.asarray(samples["theta"])
    m, s = th.mean(0), th.std(0)
    assert np.all(np.abs(m - beta) < 5 * s + 0.02), (m, beta, s)
