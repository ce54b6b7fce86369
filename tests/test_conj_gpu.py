"""Scalar conjugate updates (conj.cu through ab_conj_scalar) against the
FP64 oracle, whose restatement equals the reference's samplers bit for bit
(test_oracle_cpu.py), plus posterior moments, error handling and
checkpoint / resume."""
import os
import sys

import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N
from augurv2_b200.conj import KINDS, ScalarConj
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
import make_golden as M  # noqa: E402


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


def _conj(kind_name, off, x, aux, h0, h1, h2, seed, it):
    aux_g = None if aux is None else (off, aux)
    s = ScalarConj(kind_name, (off, x), h0, h1, h2=h2, aux=aux_g, seed=seed, iter0=it)
    s.step()
    torch.cuda.synchronize()
    ssum, saux = s.stats()
    return s.get(), ssum, saux


@pytest.mark.parametrize("kind", range(7))
def test_matches_oracle(orc, kind):
    name = M.CONJ_KINDS[kind]
    off, x, aux, h0, h1, h2 = M.conj_inputs(name, 100 + kind)
    for seed, it in ((23, 0), (23, 5), (7, 1000)):
        out, ssum, saux = _conj(name, off, x, aux, h0, h1, h2, seed, it)
        w_out, w_sum, w_aux = orc.conj_scalar(kind, off, x, h0, h1, h2, aux=aux, seed=seed, it=it)
        if kind <= 2:   # integer statistics: exact
            np.testing.assert_array_equal(ssum, w_sum)
        else:           # a fixed-order warp sum against the sequential one
            np.testing.assert_allclose(ssum, w_sum, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(saux, w_aux, rtol=1e-12, atol=0)
        np.testing.assert_allclose(out, w_out, rtol=1e-10, atol=1e-13)


def test_golden_first_draws(orc):
    g = np.load(os.path.join(GOLD, "conj_scalar.npz"))
    for kind, name in enumerate(M.CONJ_KINDS):
        off, x, aux, h0, h1, h2 = M.conj_inputs(name, 100 + kind)
        out, _, _ = _conj(name, off, x, aux, h0, h1, h2, 23, 5)
        np.testing.assert_allclose(out, g["%s_it5_out" % name], rtol=1e-10, atol=1e-13)


# (kind, observations of one group, h0, h1, h2, aux, posterior mean)
def _posterior_cases():
    rng = np.random.default_rng(3)
    yb = (rng.random(50) < 0.3).astype(float)
    yg = rng.geometric(0.4, 40) - 1.0
    yp = rng.poisson(3.0, 30).astype(float)
    ye = rng.exponential(0.5, 25)
    ys = rng.gamma(2.0, 0.25, 20)
    ai = rng.uniform(0.5, 4.0, 20)
    yi = 1.0 / rng.gamma(3.0, 0.5, 20)
    yn = rng.normal(1.5, 2.0, 15)
    return [
        ("beta_bernoulli", yb, 0.7, 1.3, None, None, (0.7 + yb.sum()) / (2.0 + len(yb))),
        ("beta_geometric", yg, 0.7, 1.3, None, None, (0.7 + len(yg)) / (2.0 + len(yg) + yg.sum())),
        ("gamma_poisson", yp, 0.7, 1.3, None, None, (0.7 + yp.sum()) / (1.3 + len(yp))),
        ("gamma_exponential", ye, 0.7, 1.3, None, None, (0.7 + len(ye)) / (1.3 + ye.sum())),
        ("gamma_gammashape", ys, 0.7, 1.3, None, ai, (0.7 + ai.sum()) / (1.3 + ys.sum())),
        ("gamma_invgamma", yi, 0.7, 1.3, None, ai, (0.7 + ai.sum()) / (1.3 + (1.0 / yi).sum())),
        ("normal_normalmean", yn, -0.5, 1.3, 4.0, None,
         (-0.5 / 1.3 + yn.sum() / 4.0) / (1.0 / 1.3 + len(yn) / 4.0)),
    ]


@pytest.mark.parametrize("case", _posterior_cases(), ids=lambda c: c[0])
def test_posterior_mean(case):
    """4096 copies of one group draw iid from its posterior: their mean is
    the analytic posterior mean within 5 standard errors."""
    name, y, h0, h1, h2, aux, mean = case
    G = 4096
    groups = [y] * G
    s = ScalarConj(name, groups, h0, h1, h2=h2, aux=None if aux is None else [aux] * G, seed=11)
    v = s.step().cpu().numpy()
    assert np.all(np.isfinite(v))
    assert abs(v.mean() - mean) < 5 * v.std() / np.sqrt(G)


def test_errors_and_nan():
    L = N.lib()
    off = torch.zeros(2, dtype=torch.int32, device="cuda")
    h = torch.ones(1, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = N.stream_ptr()
    assert L.ab_conj_scalar(7, 1, N.ptr(off), None, None, N.ptr(h), N.ptr(h), None, 0, None, None,
                            N.ptr(out), 0, 0, st) == N.AB_ERR_ARG
    assert L.ab_conj_scalar(KINDS["gamma_invgamma"], 1, N.ptr(off), None, None, N.ptr(h), N.ptr(h), None,
                            0, None, None, N.ptr(out), 0, 0, st) == N.AB_ERR_ARG
    assert L.ab_conj_scalar(KINDS["normal_normalmean"], 1, N.ptr(off), None, None, N.ptr(h), N.ptr(h), None,
                            0, None, None, N.ptr(out), 0, 0, st) == N.AB_ERR_ARG
    assert L.ab_conj_scalar(0, 0, None, None, None, None, None, None, 0, None, None, None, 0, 0, st) == N.AB_OK
    # a posterior outside the sampler's domain gives NaN, not a long loop
    s = ScalarConj("gamma_poisson", [[1.0, 2.0], []], 0.5, -3.0)
    v = s.step().cpu().numpy()
    assert np.isnan(v).all()
    s = ScalarConj("beta_bernoulli", [[1.0], [0.0]], np.array([1.0, float("nan")]), 1.0)
    v = s.step().cpu().numpy()
    assert np.isfinite(v[0]) and np.isnan(v[1])


def test_checkpoint_resume(tmp_path):
    y = [np.arange(5.0), np.ones(3)]
    a = ScalarConj("gamma_poisson", y, 1.0, 1.0, seed=4)
    a.step(5)
    b = ScalarConj("gamma_poisson", y, 1.0, 1.0, seed=4)
    b.step(2)
    b.save(str(tmp_path / "c.pt"))
    c = ScalarConj("gamma_poisson", y, 1.0, 1.0, seed=4)
    c.load(str(tmp_path / "c.pt"))
    c.step(3)
    assert torch.equal(a.value, c.value) and a.iteration == c.iteration
