"""GPU parity of the HLR log-density / gradient and of the HMC, NUTS, MWG and
reflective-slice transitions against the CPU oracle (itself pinned to the reference's own
kernels).

Tolerances: the data terms run in FP32 with compensated sums, so block
log-densities agree with the FP64 oracle within 1e-5 relative and each
gradient component within 1e-5 of the scale sum_n |r_n x_nk| (plus the prior
term); transitions start from the same state and substreams and agree to
1e-4 relative when the accept decision (a comparison of nearly equal
binary64 values, which FP32 data terms can flip) agrees.
"""
import numpy as np
import pytest
import torch

from augurv2_b200 import hlr as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


def make(N, D, seed, has_b, vprior, compat, x_dtype="f32"):
    X, y, beta, s2 = O.hlr_synthetic(N, D, seed, has_b=has_b)
    if x_dtype == "bf16":
        X = torch.as_tensor(X, dtype=torch.float32).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)
    om = O.HlrModel(X, y, has_b=has_b, vprior=vprior, compat=compat)
    gd = H.HlrData(X, y, has_b=has_b, vprior=vprior, compat=compat, x_dtype=x_dtype)
    return X, y, beta, s2, om, gd


@pytest.mark.parametrize("N,D,has_b,vprior,compat,xd", [
    (1000, 10, False, "invgamma", True, "f32"),
    (777, 33, True, "exponential", True, "f32"),
    (2500, 300, True, "exponential", False, "f32"),
    (3000, 64, False, "invgamma", False, "bf16"),
    (5, 1, True, "exponential", True, "f32"),
])
def test_ll_grad_matches_fp64_oracle(orc, N, D, has_b, vprior, compat, xd):
    X, y, beta, s2, om, gd = make(N, D, 3, has_b, vprior, compat, xd)
    rng = np.random.default_rng(1)
    C = 6
    pars = np.zeros((C, D + 2))
    pars[:, :D] = beta + 0.3 * rng.standard_normal((C, D))
    pars[:, D] = 0.2 * rng.standard_normal(C) if has_b else 0.0
    pars[:, D + 1] = 0.5 + rng.random(C)
    blocks = [list(range(D)), [D + 1], [D + 1] + ([D] if has_b else []) + list(range(D))]
    if has_b:
        blocks.append([D])
    for idx in blocks:
        ll, g = H.ll_grad(gd, pars, idx)
        for c in range(C):
            l_ref = O.hlr_ll(orc, om, pars[c], idx)
            g_ref = O.hlr_grad(orc, om, pars[c], idx)
            assert abs(ll[c] - l_ref) <= 1e-5 * abs(l_ref) + 1e-9, (idx[:3], c, ll[c], l_ref)
            t = X @ pars[c, :D] + (pars[c, D] if has_b else 0.0)
            r = np.abs(y - 1.0 / (1.0 + np.exp(-t)))
            scale_th = np.abs(X).T @ r + np.abs(pars[c, :D]) / pars[c, D + 1]
            for j, i in enumerate(idx):
                if i < D:
                    tol = 1e-5 * scale_th[i] + 1e-9
                elif i == D:
                    tol = 1e-5 * (r.sum() + abs(pars[c, D]) / pars[c, D + 1]) + 1e-9
                else:
                    tol = 1e-9 * max(1.0, abs(g_ref[j]))
                assert abs(g[c, j] - g_ref[j]) <= tol, (idx[:3], c, j, g[c, j], g_ref[j])


def run_one(gd, sched, par, it, seed, C=1):
    ch = H.HlrChains(gd, sched, C=C, init=par, seed=seed, iter0=it)
    ch.run(1)
    return ch.state(), ch.stats.cpu().numpy()


@pytest.mark.parametrize("has_b,vprior,block", [(False, "invgamma", ["theta"]),
                                                (True, "exponential", ["v", "b", "theta"])])
def test_hmc_transition_matches_oracle(orc, has_b, vprior, block):
    X, y, beta, s2, om, gd = make(1000, 10, 4, has_b, vprior, True)
    D = 10
    idx = H.block_indices(block, D)
    par = np.concatenate([beta, [0.1 if has_b else 0.0], [max(s2, 0.5)]])
    agree = 0
    for it in range(8):
        p_ref = par.copy()
        acc, L, prop = O.hlr_hmc(orc, om, p_ref, idx, 0.1, 0.01, 11, it)
        got, st = run_one(gd, [{"kind": "HMC", "block": block, "simlen": 0.1, "eps": 0.01}], par, it, 11)
        if int(st[0, 0, 0]) == acc:
            agree += 1
            np.testing.assert_allclose(got[0], p_ref, rtol=1e-4, atol=1e-6)
        par = p_ref
    assert agree >= 7


def test_hmc_many_chains_distinct_streams(orc):
    X, y, beta, s2, om, gd = make(400, 5, 6, False, "invgamma", True)
    D = 5
    par = np.concatenate([beta, [0.0], [1.0]])
    C = 16
    ch = H.HlrChains(gd, [{"kind": "HMC", "block": ["theta"], "simlen": 0.2, "eps": 0.02}], C=C, init=par, seed=5)
    ch.run(1)
    got = ch.state()
    idx = list(range(D))
    for c in range(0, C, 5):
        p_ref = par.copy()
        acc, L, prop = O.hlr_hmc(orc, om, p_ref, idx, 0.2, 0.02, 5, 0, chain=c)
        np.testing.assert_allclose(got[c], p_ref, rtol=1e-4, atol=1e-6)
    assert len({tuple(np.round(r, 12)) for r in got}) > 1


def test_nuts_transition_matches_oracle(orc):
    X, y, beta, s2, om, gd = make(300, 4, 8, True, "exponential", True)
    D = 4
    block = ["v", "b", "theta"]
    idx = H.block_indices(block, D)
    par = np.concatenate([beta, [0.1], [max(s2, 0.5)]])
    agree = 0
    for it in range(8):
        p_ref = par.copy()
        depth, leaves, ovf = O.hlr_nuts(orc, om, p_ref, idx, 0.05, 13, it, max_depth=10)
        got, st = run_one(gd, [{"kind": "NUTS", "block": block, "eps": 0.05, "max_depth": 10}], par, it, 13)
        if int(st[0, 0, 1]) == depth and np.allclose(got[0], p_ref, rtol=1e-4, atol=1e-6):
            agree += 1
        par = p_ref
    assert agree >= 7


def test_mwg_matches_oracle(orc):
    X, y, beta, s2, om, gd = make(500, 6, 9, True, "exponential", True)
    D = 6
    par = np.concatenate([beta, [0.3], [1.3]])
    for which, name in [(D + 1, "v"), (D, "b")]:
        p = par.copy()
        for it in range(6):
            p_ref = p.copy()
            acc = O.hlr_mwg(orc, om, p_ref, which, 0.5, 21, it)
            got, st = run_one(gd, [{"kind": "MWG", "var": name, "scale": 0.5}], p, it, 21)
            assert int(st[0, 0, 0]) == acc
            np.testing.assert_allclose(got[0], p_ref, rtol=1e-12)
            p = p_ref


@pytest.mark.parametrize("block,simlen,eps", [(["theta"], 0.5, 0.05), (["v", "b", "theta"], 1.0, 0.08)])
def test_rslice_matches_oracle(orc, block, simlen, eps):
    """Reflective slice (h_augur_mcmc_refl_slice): the same move or stay,
    the same number of reflections, and the same end point (1e-4) as the
    oracle, itself equal to the reference's kernel bit for bit."""
    X, y, beta, s2, om, gd = make(400, 5, 17, True, "exponential", True)
    D = 5
    idx = H.block_indices(block, D)
    par = np.concatenate([beta, [0.1], [max(s2, 0.5)]])
    agree, refl_total = 0, 0
    for it in range(10):
        p_ref = par.copy()
        moved, L, refl = O.hlr_rslice(orc, om, p_ref, idx, simlen, eps, 19, it)
        got, st = run_one(gd, [{"kind": "RSlice", "block": block, "simlen": simlen, "eps": eps}], par, it, 19)
        refl_total += refl
        if int(st[0, 0, 0]) == moved and int(st[0, 0, 2]) == refl and \
                np.allclose(got[0], p_ref, rtol=1e-4, atol=1e-6):
            agree += 1
        par = p_ref
    assert agree >= 9
    assert refl_total > 0


def test_schedule_composition_runs():
    X, y, beta, s2, om, gd = make(800, 8, 10, True, "exponential", True)
    sched = [{"kind": "MWG", "var": "v", "scale": 1.0}, {"kind": "MWG", "var": "b", "scale": 1.0},
             {"kind": "HMC", "block": ["theta"], "simlen": 0.5, "eps": 0.05}]
    ch = H.HlrChains(gd, sched, C=8, init=np.concatenate([beta, [0.0], [1.0]]), seed=1)
    ch.run(20)
    s = ch.state()
    assert np.isfinite(s).all() and (s[:, 9] > 0).all()
    st = ch.stats.cpu().numpy()
    assert (st[:, 2, 0] > 0).all()
