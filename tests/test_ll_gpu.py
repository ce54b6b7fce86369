"""Whole-model log densities (augur_get_curr_ll's ll_mod), held-out
predictive log-likelihoods and dethlr's deterministic bias on the device,
against the CPU oracle.

Tolerance: the device sums in a different order from the oracle's
sequential loops, so a value may differ by rounding: |device - oracle| <=
1e-12 * (sum of the absolute values of the terms)."""
import numpy as np
import pytest
import torch

from augurv2_b200.gmm import GmmGibbs
from augurv2_b200.hlr import HlrChains, HlrData
from augurv2_b200.lda import LdaGibbs, synthetic_corpus
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL = 1e-12


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


def _lda_state(seed, K=20, V=300, D=50):
    off, w = synthetic_corpus(K, V, D, 40, 0.2, 0.05, seed=seed)
    s = LdaGibbs(K, V, off, w, 0.2, 0.05, seed=seed)
    s.sweep(3)
    return off, w, s


@pytest.mark.parametrize("seed,K,V,D", [(1, 20, 300, 50), (2, 50, 10000, 2000), (3, 3, 7, 5)])
def test_lda_ll_mod_matches_oracle(orc, seed, K, V, D):
    off, w, s = _lda_state(seed, K, V, D)
    theta, phi, z = s.state()
    alpha, beta = np.full(K, 0.2), np.full(V, 0.05)
    ref = orc.lda_ll_mod(off, w, z, alpha, beta, theta, phi)
    doc = np.repeat(np.arange(D), np.diff(off))
    scale = (np.abs((alpha - 1) * np.log(theta)).sum() + np.abs((beta - 1) * np.log(phi)).sum()
             + np.abs(np.log(theta[doc, z])).sum() + np.abs(np.log(phi[z, w])).sum())
    got = s.ll_mod()
    assert abs(got - ref) <= REL * scale, (got, ref, scale)
    s.close()


def test_lda_pred_ll_matches_oracle(orc):
    K, V, D = 30, 500, 80
    off, w, s = _lda_state(7, K, V, D)
    rng = np.random.default_rng(3)
    lens = rng.integers(0, 12, size=D)
    lens[::9] = 0                               # documents without held-out tokens
    ho_off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ho_w = rng.integers(0, V, size=ho_off[-1]).astype(np.int32)
    theta, phi, _ = s.state()
    ref = orc.lda_pred_ll(ho_off, ho_w, theta, phi)
    got = s.pred_ll((ho_off, ho_w))
    assert abs(got - ref) <= REL * 40 * len(ho_w), (got, ref)
    # the per-document list form gives the same value
    docs = [ho_w[ho_off[d]:ho_off[d + 1]] for d in range(D)]
    assert s.pred_ll(docs) == got
    s.close()


@pytest.mark.parametrize("shared,N_,K,d", [(False, 3000, 4, 5), (True, 2000, 3, 2), (False, 20000, 16, 32)])
def test_gmm_ll_mod_and_pred_ll_match_oracle(orc, shared, N_, K, d):
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, seed=d)
    if shared:
        g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), pis=pis, covs=covs[0], mu=mus, z=z, seed=2)
        om = O.GmmModel(Y.astype(np.float64), K, np.zeros(d), 25 * np.eye(d), True)
    else:
        g = GmmGibbs(Y, K, np.zeros(d), 25 * np.eye(d), alpha=np.full(K, 1.5), df=d + 2, scale0=np.eye(d),
                     mu=mus, cov=covs, pis=pis, z=z, seed=2)
        om = O.GmmModel(Y.astype(np.float64), K, np.zeros(d), 25 * np.eye(d), False, alpha=np.full(K, 1.5),
                        df=d + 2, scale0=np.eye(d))
    g.sweep(2)
    st = g.state()
    cov = g.cov.cpu().numpy()[0] if shared else st["cov"]
    ref = O.gmm_ll_mod(orc, om, st["pis"], st["mu"], cov, st["z"])
    got = g.ll_mod()
    # scale: the data term dominates; |log N| per point is bounded by a few hundred at these d
    scale = abs(ref) + N_ * (d + 10)
    assert abs(got - ref) <= REL * scale, (got, ref)
    Yt = O.gmm_synthetic(500, K, d, seed=d + 100)[0]
    ref = O.gmm_pred_ll(orc, Yt.astype(np.float64), st["pis"], st["mu"], cov, shared_cov=shared)
    got = g.pred_ll(Yt)
    assert abs(got - ref) <= REL * (abs(ref) + 500 * (d + 10)), (got, ref)


def test_hlr_det_bias_matches_fp64(orc):
    rng = np.random.default_rng(4)
    N_, D, C = 700, 9, 5
    X = rng.standard_normal((N_, D)).astype(np.float32)
    y = (rng.random(N_) < 0.5).astype(np.int32)
    for x_dtype in ("f32", "bf16"):
        data = HlrData(X, y, has_b=True, vprior="exponential", x_dtype=x_dtype)
        init = np.concatenate([rng.standard_normal((C, D)), rng.standard_normal((C, 1)), np.ones((C, 1))], 1)
        ch = HlrChains(data, [{"kind": "HMC", "block": ["theta"], "simlen": 0.1, "eps": 0.05}], C=C, init=init)
        got = ch.det_bias().cpu().numpy()
        Xd = data.X.float().cpu().numpy().astype(np.float64)
        t = init[:, :D] @ Xd.T + init[:, D:D + 1]
        np.testing.assert_allclose(got, 1.0 / (1.0 + np.exp(-t)), rtol=1e-13, atol=1e-15)
