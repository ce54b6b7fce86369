"""Many model instances in one launch per stage: the grouped HLR pass
(ab_hlrg_*) and the grouped NUTS advance (ab_nutsg_*, NutsGroup).

Contracts:
  fused pass (every D <= 256)  logp and grad within the FP64-oracle
         tolerance of the batched pass (log density 1e-5 of sum_n |term_n|,
         gradient 1e-5 of |g| + sum_n |r_n x_nd|), and an instance's numbers
         identical alone and in any group;
  two-GEMM grouped pass (some D > 256)  equal to each instance's own
         ab_hlrb_logp_grad bit for bit;
  NUTS   every instance's draws, depths and proposals equal a group of that
         instance alone run for the same number of rounds, and the FP64
         oracle's NUTS draws (cbits/augur_mcmclib.h:575-776)."""
import ctypes as C

import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N
from augurv2_b200 import hlrb as H
from oracle import batched as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(3000, 64, 40, "student_t"), (1000, 16, 3, "normal"), (2500, 200, 130, "student_t"),
          (777, 520, 9, "normal"), (64, 8, 1, "student_t"), (20000, 128, 256, "student_t"),
          (1498, 256, 512, "normal")]


def _data(N_, D, seed, prior="student_t", scale=0.3):
    rs = np.random.default_rng(seed)
    X = torch.as_tensor(rs.standard_normal((N_, D)), dtype=torch.float32).to(torch.bfloat16)
    beta = rs.standard_normal(D) * scale
    t = X.double().numpy() @ beta
    y = (rs.random(N_) < 1 / (1 + np.exp(-t))).astype(np.int32)
    return H.HlrbData(X, y, prior=prior, nu=3.0, scale=1.0, var=2.0), X.double().numpy(), y


class _Group:
    def __init__(self, datas, Cs):
        n = len(datas)
        self.h = C.c_void_p()
        models = (H.HlrbModelC * n)(*[d.c for d in datas])
        N.check(N.lib().ab_hlrg_create(n, models, (C.c_int * n)(*Cs), C.byref(self.h)), "ab_hlrg_create")

    def bind(self, i, th, lp, g):
        N.check(N.lib().ab_hlrg_bind(self.h, i, N.ptr(th), th.shape[1], N.ptr(lp), N.ptr(g), g.shape[1]),
                "ab_hlrg_bind")

    def active(self, mask):
        a = (C.c_int * len(mask))(*[int(m) for m in mask])
        N.check(N.lib().ab_hlrg_set_active(self.h, a, N.stream_ptr()), "ab_hlrg_set_active")

    def run(self, err):
        N.check(N.lib().ab_hlrg_logp_grad(self.h, N.ptr(err), N.stream_ptr()), "ab_hlrg_logp_grad")

    def fused(self):
        return N.lib().ab_hlrg_fused(self.h) == 1

    def close(self):
        N.lib().ab_hlrg_destroy(self.h)


def _fp64_check(X64, y, d, th, lp, g):
    lp64, g64, scale = B.hlr_logp_grad(X64, y, th.double().cpu().numpy(), d.prior, d.pa, d.pb)
    t = th.double().cpu().numpy() @ X64.T
    term_scale = (np.abs(y * t) + np.logaddexp(0, t)).sum(-1)
    e_lp = np.abs(lp.cpu().numpy() - lp64) / term_scale
    gd = g.cpu().numpy().astype(np.float64)
    e_g = np.abs(gd - g64) / (np.abs(g64) + scale)
    assert e_lp.max() <= 1e-5 and e_g.max() <= 1e-5, (e_lp.max(), e_g.max())


FUSED = [(3000, 64, 40, "student_t"), (1000, 16, 3, "normal"), (2500, 200, 130, "student_t"),
         (64, 8, 1, "student_t"), (20000, 128, 256, "student_t"), (1498, 256, 512, "normal"),
         (50, 24, 7, "normal"), (70000, 256, 129, "student_t")]


def _run_group(datas, ths, mask=None):
    g = _Group(datas, [t.shape[0] for t in ths])
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lps = [torch.full((t.shape[0],), float("nan"), dtype=torch.float64, device="cuda") for t in ths]
    gs = [torch.full(t.shape, float("nan"), dtype=torch.float32, device="cuda") for t in ths]
    for i, t in enumerate(ths):
        g.bind(i, t, lps[i], gs[i])
    g.active(mask if mask is not None else [1] * len(ths))
    g.run(err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    fused = g.fused()
    g.close()
    return lps, gs, fused


def test_fused_pass_matches_fp64_and_is_independent_of_the_group():
    raw = [_data(n, d, seed=7 * n + d + c, prior=p) for n, d, c, p in FUSED]
    datas = [r[0] for r in raw]
    rs = np.random.default_rng(3)
    ths = [torch.as_tensor(rs.standard_normal((c, d.D)) * 0.3, dtype=torch.float32, device="cuda")
           for d, (_, _, c, _) in zip(datas, FUSED)]
    lps, gs, fused = _run_group(datas, ths)
    assert fused
    for (d, X64, y), th, lp, g in zip(raw, ths, lps, gs):
        _fp64_check(X64, y, d, th, lp, g)
    # each instance alone gives the same bits, and so does a subset
    for i in (0, 5, 7):
        lp1, g1, _ = _run_group([datas[i]], [ths[i]])
        assert torch.equal(lp1[0], lps[i]) and torch.equal(g1[0], gs[i])
    mask = [i % 3 != 1 for i in range(len(datas))]
    lp2, g2, _ = _run_group(datas, ths, mask)
    for m, a, b, ga, gb in zip(mask, lp2, lps, g2, gs):
        if m:
            assert torch.equal(a, b) and torch.equal(ga, gb)
        else:
            assert torch.isnan(a).all() and torch.isnan(ga).all()


def test_two_gemm_grouped_pass_equals_each_instance_bit_for_bit():
    datas = [_data(n, d, seed=n + d + c, prior=p)[0] for n, d, c, p in SHAPES]
    Cs = [c for _, _, c, _ in SHAPES]
    rs = np.random.default_rng(0)
    g = _Group(datas, Cs)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ths = [torch.as_tensor(rs.standard_normal((c, d.D)) * 0.3, dtype=torch.float32, device="cuda")
           for d, c in zip(datas, Cs)]
    lps = [torch.full((c,), float("nan"), dtype=torch.float64, device="cuda") for c in Cs]
    gs = [torch.full((c, d.D), float("nan"), dtype=torch.float32, device="cuda") for d, c in zip(datas, Cs)]
    for i in range(len(datas)):
        g.bind(i, ths[i], lps[i], gs[i])
    g.active([1] * len(datas))
    g.run(err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert not g.fused()          # D = 520: the two-GEMM grouped pass
    for d, th, lp, gr in zip(datas, ths, lps, gs):
        lp0, g0 = d.logp_grad(th)
        assert torch.equal(lp, lp0) and torch.equal(gr, g0)
    # a subset: the others' outputs are left alone, the active ones follow new inputs
    mask = [i % 2 == 0 for i in range(len(datas))]
    for i in range(len(datas)):
        ths[i].copy_(torch.randn_like(ths[i]) * 0.2)
        lps[i].fill_(float("nan"))
        gs[i].fill_(float("nan"))
    g.active(mask)
    g.run(err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for m, d, th, lp, gr in zip(mask, datas, ths, lps, gs):
        if m:
            lp0, g0 = d.logp_grad(th)
            assert torch.equal(lp, lp0) and torch.equal(gr, g0)
        else:
            assert torch.isnan(lp).all() and torch.isnan(gr).all()
    g.close()


def test_grouped_pass_argument_errors():
    d, _, _ = _data(500, 16, seed=1)
    h = C.c_void_p()
    L = N.lib()
    models = (H.HlrbModelC * 1)(d.c)
    assert L.ab_hlrg_create(0, models, (C.c_int * 1)(4), C.byref(h)) == N.AB_ERR_ARG
    assert L.ab_hlrg_create(1, models, (C.c_int * 1)(0), C.byref(h)) == N.AB_ERR_ARG
    N.check(L.ab_hlrg_create(1, models, (C.c_int * 1)(4), C.byref(h)), "ab_hlrg_create")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    # unbound instance made active, and a pass before any set_active, are refused
    assert L.ab_hlrg_set_active(h, (C.c_int * 1)(1), N.stream_ptr()) == N.AB_ERR_STATE
    assert L.ab_hlrg_logp_grad(h, N.ptr(err), N.stream_ptr()) == N.AB_ERR_STATE
    assert "set_active" in N.last_error()
    L.ab_hlrg_destroy(h)


def _instances(specs, C_, depth, hist_cap=24):
    out = []
    for i, (N_, D, eps) in enumerate(specs):
        d, X64, y = _data(N_, D, seed=40 + i, prior="normal")
        init = (np.random.default_rng(i).standard_normal((C_, D)) * 0.1).astype(np.float32)
        out.append((d, eps, init, 3 + i))
    return [H.BatchedNuts(d, C_, eps=eps, max_depth=depth, seed=s, init=init, hist_cap=hist_cap)
            for d, eps, init, s in out], out


def test_nuts_group_equals_each_instance_run_alone():
    specs = [(300, 8, 0.08), (2000, 16, 0.03), (800, 64, 0.03), (5000, 256, 0.01)]
    insts, raw = _instances(specs, 6, depth=5)
    grp = H.NutsGroup(insts)
    ran = grp.run(min_draws=5, max_rounds=500, block=10)
    for s, r in zip(insts, ran):
        assert 0 < r <= 500
        assert s.info()[:, 0].min() >= 5
    # instances left the launches at different rounds
    assert len(set(ran)) > 1
    for (d, eps, init, seed), s, r in zip(raw, insts, grp.rounds):
        solo = H.BatchedNuts(d, 6, eps=eps, max_depth=5, seed=seed, init=init, hist_cap=24)
        alone = H.NutsGroup([solo])
        alone.step(r)
        alone.close()
        assert torch.equal(solo.thprop, s.thprop)
        assert torch.equal(solo.hist, s.hist) and torch.equal(solo.hist_depth, s.hist_depth)
        np.testing.assert_array_equal(solo.info(), s.info())
    grp.reset()
    assert all(s.info()[:, 0].max() == 0 for s in insts)
    ran2 = grp.run(min_draws=3, max_rounds=500, block=10)
    assert all(s.info()[:, 0].min() >= 3 for s in insts) and all(r > 0 for r in ran2)
    grp.close()


def test_nuts_group_matches_fp64_oracle_nuts():
    """The reference's NUTS (FP64 oracle restatement of h_augur_mcmc_nuts,
    cbits/augur_mcmclib.h:575-776) fed the same Philox streams, against an
    instance advanced by the grouped launches next to a second instance."""
    o = O.Oracle("oracle")
    N_, D, C_, v, eps, seed, depth = 400, 8, 5, 2.0, 0.05, 13, 6
    _, X64, y = _data(N_, D, seed=31, prior="normal")
    d = H.HlrbData(torch.as_tensor(X64, dtype=torch.float32).to(torch.bfloat16), y, prior="normal", var=v)
    rs = np.random.default_rng(4)
    init = (rs.standard_normal((C_, D)) * 0.3).astype(np.float32)
    nuts = H.BatchedNuts(d, C_, eps=eps, max_depth=depth, seed=seed, init=init, hist_cap=32)
    other, _ = _instances([(3000, 64, 0.02)], 7, depth=depth)
    grp = H.NutsGroup([nuts] + other)
    grp.run(min_draws=6, max_rounds=400, block=20)
    got = nuts.draws()
    depths = nuts.hist_depth.cpu().numpy()
    assert got.shape[0] >= 6
    m = O.HlrModel(X64, y, has_b=False, vprior="invgamma")
    for c in range(C_):
        par = np.zeros(D + 2)
        par[:D] = init[c]
        par[D + 1] = v
        for it in range(6):
            dep, leaves, ovf = O.hlr_nuts(o, m, par, list(range(D)), float(np.float32(eps)), seed, it, chain=c,
                                          comp=0, max_depth=depth)
            assert dep == depths[c, it], (c, it, dep, depths[c, it])
            np.testing.assert_allclose(got[it, c], par[:D], rtol=2e-4, atol=2e-5)
    grp.close()
