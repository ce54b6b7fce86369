"""Divergence counting of the HMC and NUTS samplers.

A transition is divergent when its energy error H_end - H_start exceeds
AB_DIVERGENCE_DH (1000, the reference NUTS's deltaMax of
cbits/augur_mcmclib.h:152) or is not finite; for NUTS, an iteration is
divergent when one of its leaves falls below the slice level by more than
that.  The batched HMC count is checked against the FP64 oracle's energy
errors for the same Philox draws; the per-chain engine and the batched NUTS
count divergences at a step size far too large for the posterior and none
at a small one.
"""
import numpy as np
import pytest
import torch

from augurv2_b200 import hlr as HL
from augurv2_b200 import hlrb as H
from oracle import batched as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
BOUND = 1000.0


def _data(N, D, seed):
    rs = np.random.default_rng(seed)
    X = torch.as_tensor(rs.standard_normal((N, D)), dtype=torch.float32).to(torch.bfloat16)
    t = X.double().numpy() @ (rs.standard_normal(D) * 0.3)
    y = (rs.random(N) < 1 / (1 + np.exp(-t))).astype(np.int32)
    return H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0), X.double().numpy(), y


@pytest.mark.parametrize("eps", [0.01, 0.08, 0.6])
def test_batched_hmc_divergences_match_fp64_energy_errors(eps):
    o = O.Oracle("oracle")
    d, X64, y = _data(600, 16, seed=5)
    C, L, jit, seed = 24, 4, 0.2, 3
    init = np.random.default_rng(1).standard_normal((C, 16)) * 0.2
    hmc = H.BatchedHmc(d, C, L=L, eps=eps, jitter=jit, seed=seed, init=init)
    th = hmc.theta.double().cpu().numpy()
    lp64, g64, _ = B.hlr_logp_grad(X64, y, th, d.prior, d.pa, d.pb)
    expect, near = 0, 0
    for it in range(3):
        hmc.run(1)
        th, g64, lp64, acc, dH = B.hmc_iteration(o, X64, y, th, g64, lp64, float(np.float32(eps)),
                                                 float(np.float32(jit)), L, seed, it, d.prior, d.pa, d.pb)
        div = ~(dH > -BOUND)
        expect += int(div.sum())
        near += int((np.abs(dH + BOUND) < 0.01 * BOUND).sum())
        # the chains stay together with the oracle (same accept decisions)
        np.testing.assert_allclose(hmc.theta.double().cpu().numpy(), th, rtol=1e-4, atol=1e-5)
    got = hmc.divergences()
    assert abs(got - expect) <= near, (got, expect, near)
    if eps == 0.01:
        assert got == 0
    if eps == 0.6:
        assert got > 0


def test_per_chain_engine_counts_divergences():
    rs = np.random.default_rng(2)
    N_, D = 800, 6
    X, y, beta, s2, om, gd = _hlr_problem(rs, N_, D)
    for eps, expect_some in ((0.002, False), (0.5, True)):
        sched = [{"kind": "HMC", "block": ["theta"], "simlen": 10 * eps, "eps": eps},
                 {"kind": "NUTS", "block": ["theta"], "eps": eps, "max_depth": 6}]
        ch = HL.HlrChains(gd, sched, C=8, init=np.concatenate([beta, [0.0], [s2]]), seed=4)
        ch.run(5)
        div = ch.divergences()
        assert div.shape == (2,)
        if expect_some:
            assert div[0] > 0 and div[1] > 0, div
        else:
            assert div.sum() == 0, div
        # a divergent HMC transition is never accepted
        st = ch.stats.cpu().numpy()
        assert (st[:, 0, 0] + st[:, 0, 4] <= 5).all()


def test_batched_nuts_counts_divergences():
    d, X64, y = _data(2000, 8, seed=9)
    init = np.random.default_rng(0).standard_normal((16, 8)).astype(np.float32) * 0.1
    small = H.BatchedNuts(d, 16, eps=0.005, max_depth=6, seed=2, init=init, hist_cap=16)
    small.run(200)
    assert small.divergences() == 0
    big = H.BatchedNuts(d, 16, eps=1.0, max_depth=6, seed=2, init=init, hist_cap=16)
    big.run(60)
    inf = big.info()
    assert big.divergences() > 0
    assert (inf[:, 6] <= inf[:, 0]).all()      # at most one per iteration


def _hlr_problem(rs, N_, D):
    X = rs.standard_normal((N_, D))
    beta = rs.standard_normal(D) * 0.5
    y = (rs.random(N_) < 1 / (1 + np.exp(-(X @ beta)))).astype(np.int32)
    gd = HL.HlrData(X.astype(np.float32), y, has_b=False, vprior="invgamma")
    om = O.HlrModel(X.astype(np.float32).astype(np.float64), y, has_b=False, vprior="invgamma")
    return X, y, beta, 1.0, om, gd
