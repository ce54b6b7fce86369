"""Batched HLR on the tensor cores against the FP64 oracle.

Tolerances (written here, per the FP32 data-pass contract):
  log density   |logp - logp64| <= 1e-5 * sum_n |term_n| (relative to the sum's scale)
  gradient      |g - g64| <= 1e-5 * (|g64| + sum_n |r_n x_nd|) per coordinate
Transitions: the same accept decisions as the FP64 oracle fed the same Philox
draws, and end points within 1e-4 relative."""
import numpy as np
import pytest
import torch

from augurv2_b200 import hlrb as H
from oracle import batched as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _data(N, D, seed, prior="student_t", scale=0.3):
    rs = np.random.default_rng(seed)
    X = torch.as_tensor(rs.standard_normal((N, D)), dtype=torch.float32).to(torch.bfloat16)
    beta = rs.standard_normal(D) * scale
    t = X.double().numpy() @ beta
    y = (rs.random(N) < 1 / (1 + np.exp(-t))).astype(np.int32)
    d = H.HlrbData(X, y, prior=prior, nu=3.0, scale=1.0, var=2.0)
    return d, X.double().numpy(), y


def _check(d, X64, y, theta):
    th = torch.as_tensor(theta, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lp, g = d.logp_grad(th, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    lp64, g64, scale = B.hlr_logp_grad(X64, y, th.double().cpu().numpy(), d.prior, d.pa, d.pb)
    t = th.double().cpu().numpy() @ X64.T
    term_scale = (np.abs(y * t) + np.logaddexp(0, t)).sum(-1)
    assert np.all(np.abs(lp.cpu().numpy() - lp64) <= 1e-5 * term_scale), np.max(np.abs(lp.cpu().numpy() - lp64) / term_scale)
    gd = g.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(gd - g64) <= 1e-5 * (np.abs(g64) + scale)), np.max(np.abs(gd - g64) / (np.abs(g64) + scale))
    # the log-density-only pass gives the same numbers
    lp2, _ = d.logp_grad(th, grad=False)
    np.testing.assert_array_equal(lp2.cpu().numpy(), lp.cpu().numpy())
    return lp, g


@pytest.mark.parametrize("N,D,C,prior", [(3000, 64, 40, "student_t"), (1000, 16, 3, "normal"),
                                         (2500, 200, 130, "student_t"), (777, 520, 9, "normal"),
                                         (64, 8, 1, "student_t"), (20000, 128, 256, "student_t")])
def test_logp_grad_matches_fp64(N, D, C, prior):
    d, X64, y = _data(N, D, seed=N + D + C, prior=prior)
    rs = np.random.default_rng(C)
    _check(d, X64, y, rs.standard_normal((C, D)) * 0.3)


def test_deterministic_repeat():
    d, X64, y = _data(5000, 96, seed=1)
    th = torch.randn(50, 96, device="cuda") * 0.2
    a = d.logp_grad(th)
    b = d.logp_grad(th)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_full_size_against_fp64_on_device():
    # N = 2,000,000 rows, D = 512, C = 256 chains: checked for 4 chains
    # against an FP64 product of the same bf16 data on the device.
    X, y, beta = H.synthetic(2_000_000, 512, seed=7)
    d = H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0)
    th = torch.as_tensor(beta, device="cuda").repeat(256, 1)
    th += 0.01 * torch.randn(256, 512, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lp, g = d.logp_grad(th, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    pick = [0, 77, 128, 255]
    th64 = th[pick].double()
    ll = torch.zeros(4, dtype=torch.float64, device="cuda")
    gg = torch.zeros(4, 512, dtype=torch.float64, device="cuda")
    sc = torch.zeros(4, 512, dtype=torch.float64, device="cuda")
    tscale = torch.zeros(4, dtype=torch.float64, device="cuda")
    for s in range(0, 2_000_000, 250_000):
        xs = X[s:s + 250_000].double()
        ys = y[s:s + 250_000].double()
        t = xs @ th64.T
        sp = torch.logaddexp(torch.zeros_like(t), t)
        ll += (ys[:, None] * t - sp).sum(0)
        tscale += (torch.abs(ys[:, None] * t) + sp).sum(0)
        r = ys[:, None] - torch.sigmoid(t)
        gg += r.T @ xs
        sc += r.abs().T @ xs.abs()
    pl, pg = B.prior_terms(th64.cpu().numpy(), 1, 3.0, 1.0)
    ll = ll.cpu().numpy() + pl
    gg = gg.cpu().numpy() + pg
    sc = sc.cpu().numpy()
    lpd = lp[pick].cpu().numpy()
    gd = g[pick].double().cpu().numpy()
    assert np.all(np.abs(lpd - ll) <= 1e-5 * tscale.cpu().numpy())
    assert np.all(np.abs(gd - gg) <= 1e-5 * (np.abs(gg) + sc))


def test_hmc_transitions_match_fp64_oracle():
    o = O.Oracle("oracle")
    d, X64, y = _data(600, 16, seed=11, prior="student_t")
    C, L, eps, jit, seed = 6, 4, 0.05, 0.2, 9
    rs = np.random.default_rng(3)
    init = rs.standard_normal((C, 16)) * 0.2
    hmc = H.BatchedHmc(d, C, L=L, eps=eps, jitter=jit, seed=seed, init=init)
    th = hmc.theta.double().cpu().numpy()
    lp64, g64, _ = B.hlr_logp_grad(X64, y, th, d.prior, d.pa, d.pb)
    n_acc = 0
    for it in range(4):
        hmc.run(1)
        th, g64, lp64, acc, dH = B.hmc_iteration(o, X64, y, th, g64, lp64, float(np.float32(eps)), float(np.float32(jit)),
                                                 L, seed, it, d.prior, d.pa, d.pb)
        n_acc += acc.sum()
        got = hmc.theta.double().cpu().numpy()
        np.testing.assert_allclose(got, th, rtol=1e-4, atol=1e-5)
    st = hmc.s.stats.cpu().numpy()
    assert int(st[:, 0].sum()) == n_acc
    assert n_acc > 0


def test_graph_replay_equals_eager():
    d, X64, y = _data(4000, 64, seed=5)
    init = np.random.default_rng(0).standard_normal((16, 64)) * 0.1
    a = H.BatchedHmc(d, 16, L=3, eps=0.02, seed=4, init=init)
    b = H.BatchedHmc(d, 16, L=3, eps=0.02, seed=4, init=init)
    a.run(3)
    b.capture()
    b.run(3)
    torch.cuda.synchronize()
    assert torch.equal(a.theta, b.theta)


def test_batched_nuts_matches_fp64_oracle_nuts():
    # The reference's NUTS on the HLR block theta with v fixed (ighlr.rv's
    # conditional), FP64 oracle, against the batched sampler fed the same
    # Philox streams: same draws to FP32 accuracy and the same tree depths.
    o = O.Oracle("oracle")
    N_, D, C, v, eps, seed, depth = 400, 8, 5, 2.0, 0.05, 13, 6
    d, X64, y = _data(N_, D, seed=31, prior="normal")
    d = H.HlrbData(torch.as_tensor(X64, dtype=torch.float32).to(torch.bfloat16), y, prior="normal", var=v)
    rs = np.random.default_rng(4)
    init = (rs.standard_normal((C, D)) * 0.3).astype(np.float32)
    nuts = H.BatchedNuts(d, C, eps=eps, max_depth=depth, seed=seed, init=init, hist_cap=32)
    nuts.run(400)
    got = nuts.draws()
    depths = nuts.hist_depth.cpu().numpy()
    assert got.shape[0] >= 4
    m = O.HlrModel(X64, y, has_b=False, vprior="invgamma")
    for c in range(C):
        par = np.zeros(D + 2)
        par[:D] = init[c]
        par[D + 1] = v
        for it in range(min(6, got.shape[0])):
            dep, leaves, ovf = O.hlr_nuts(o, m, par, list(range(D)), float(np.float32(eps)), seed, it, chain=c,
                                          comp=0, max_depth=depth)
            assert dep == depths[c, it], (c, it, dep, depths[c, it])
            np.testing.assert_allclose(got[it, c], par[:D], rtol=2e-4, atol=2e-5)


@pytest.mark.parametrize("N,D,C", [(3000, 64, 40), (20000, 16, 130), (2500, 200, 256)])
def test_every_launch_shape_matches_fp64(N, D, C, tmp_path):
    """Every launch shape the autotuner may pick computes the same log
    density and gradient (within the FP64-oracle tolerance), and the tuner's
    pick is one of them and is reused from its cache."""
    from augurv2_b200 import autotune as T
    d, X64, y = _data(N, D, seed=N + D, prior="student_t")
    th = np.random.default_rng(C).standard_normal((C, D)) * 0.3
    cands = T.hlrb_candidates(N, D, C, torch.cuda.get_device_properties(0).multi_processor_count)
    for cand in cands:
        d.config = T.HlrbConfigC.of(cand)
        _check(d, X64, y, th)
    tuner = T.Autotuner(cache_path=str(tmp_path / "tune.json"), reps=2, warmup=1)
    d.config = None
    best = d.autotune(C, tuner=tuner)
    assert best in cands and tuner.timed == len(cands)
    _check(d, X64, y, th)
    again = T.Autotuner(cache_path=str(tmp_path / "tune.json"))
    d.config = None
    assert d.autotune(C, tuner=again) == best and again.timed == 0


def test_workspace_too_small_for_shape_is_refused():
    from augurv2_b200 import _native as Nn
    from augurv2_b200 import autotune as T
    d, X64, y = _data(50000, 16, seed=3)
    th = torch.zeros((8, 16), device="cuda")
    small = d.workspace(8, T.HlrbConfigC.of({"bwd_splits": 1}))
    with pytest.raises(Nn.AugurError):
        d.logp_grad(th, work=small, config=T.HlrbConfigC.of({"bwd_splits": 300}))


def test_nuts_pool_runs_until_every_instance_has_its_draws():
    insts = []
    for i, (N_, D, eps) in enumerate([(300, 8, 0.08), (2000, 16, 0.03), (800, 64, 0.03)]):
        d, X64, y = _data(N_, D, seed=40 + i, prior="normal")
        init = (np.random.default_rng(i).standard_normal((6, D)) * 0.1).astype(np.float32)
        insts.append(H.BatchedNuts(d, 6, eps=eps, max_depth=5, seed=3 + i, init=init, hist_cap=16))
    # the same sampler run alone, for comparison of the draws
    d0, _, _ = _data(300, 8, seed=40, prior="normal")
    solo = H.BatchedNuts(d0, 6, eps=0.08, max_depth=5, seed=3,
                         init=(np.random.default_rng(0).standard_normal((6, 8)) * 0.1).astype(np.float32), hist_cap=16)
    pool = H.NutsPool(insts, streams=2)
    ran = pool.run(min_draws=5, max_rounds=500, block=10)
    for s, r in zip(insts, ran):
        assert 0 < r <= 500
        assert s.info()[:, 0].min() >= 5
    # a pool changes only the scheduling: instance 0's draws equal a solo run's
    solo.capture()
    solo.run(pool.rounds[0] - 1)
    n = min(solo.draws().shape[0], insts[0].draws().shape[0])
    np.testing.assert_array_equal(solo.draws()[:n], insts[0].draws()[:n])
    pool.reset()
    assert all(s.info()[:, 0].max() == 0 for s in insts)
    ran2 = pool.run(min_draws=3, max_rounds=500, block=10)
    assert all(s.info()[:, 0].min() >= 3 for s in insts) and all(r > 0 for r in ran2)


def _posterior_summary(draws):
    """draws [n, C, D] -> (mean [D], sd [D], ESS [D])"""
    from augurv2_b200.diagnostics import ess
    x = np.asarray(draws, np.float64)
    flat = x.reshape(-1, x.shape[-1])
    return flat.mean(0), flat.std(0), ess(x)


def test_nuts_posterior_moments_match_exact_hmc():
    """ESS-scaled z-tests of posterior means (and a check of the sds): the
    batched NUTS, under both selection rules, against plain exact-gradient
    HMC (whose transitions equal the FP64 oracle's) on the same HLR
    posterior; both rules mix well here (ESS at least 0.2 per draw)."""
    N_, D, v = 400, 8, 2.0
    d, X64, y = _data(N_, D, seed=77, prior="normal")
    d = H.HlrbData(torch.as_tensor(X64, dtype=torch.float32).to(torch.bfloat16), y, prior="normal", var=v)
    rs = np.random.default_rng(5)
    C_ = 256
    init = (rs.standard_normal((C_, D)) * 0.5).astype(np.float32)
    w = 0.2
    eps = 0.6 / np.sqrt(N_ * w + 1.0 / v)
    out = {}
    for variant in ("standard", "reference"):
        nuts = H.BatchedNuts(d, C_, eps=eps, max_depth=8, seed=21, init=init, hist_cap=160, variant=variant)
        nuts.capture()
        pool = H.NutsPool([nuts], streams=1)
        pool.run(min_draws=40, max_rounds=20000)          # warm-up
        pool.reset()
        pool.run(min_draws=150, max_rounds=40000)
        out[variant] = _posterior_summary(nuts.draws()[:150])
    hmc = H.BatchedHmc(d, C_, L=10, eps=eps, jitter=0.1, seed=8, init=init)
    hmc.capture()
    hmc.run(100)
    rec = []
    for _ in range(300):
        hmc.run(1)
        rec.append(hmc.theta.detach().cpu().numpy().copy())
    m_h, s_h, e_h = _posterior_summary(np.stack(rec))
    for variant, (m_n, s_n, e_n) in out.items():
        z = (m_n - m_h) / np.sqrt(s_h ** 2 / e_h + s_n ** 2 / e_n)
        assert np.all(np.abs(z) < 4.5), (variant, z)
        np.testing.assert_allclose(s_n, s_h, rtol=0.15, err_msg=variant)
        assert e_n.min() > 0.2 * 150 * C_, (variant, e_n.min())
