"""The FP64 oracle of the batched HLR path, pinned to the reference's own
HLR block gradient (the generated grad_ code restated over cbits) and
checked by finite differences; the surrogate network's FP64 gradient by
finite differences."""
import numpy as np
import pytest

from oracle import batched as B
from oracle import oracle as O


def _ref():
    return O.Oracle("ref") if O.available("ref") else O.Oracle("oracle")


def test_block_gradient_equals_reference_hlr_grad():
    o = _ref()
    X, y, _, s2 = O.hlr_synthetic(300, 7, seed=3, has_b=False)
    m = O.HlrModel(X, y, has_b=False, vprior="invgamma")
    rs = np.random.default_rng(0)
    for _ in range(3):
        theta = rs.standard_normal(7) * 0.5
        par = np.concatenate([theta, [0.0, s2]])
        g_ref = O.hlr_grad(o, m, par, list(range(7)))
        _, g, _ = B.hlr_logp_grad(X, y, theta[None], prior=0, a=s2)
        np.testing.assert_allclose(g[0], g_ref, rtol=1e-12, atol=1e-12)


def test_block_log_density_equals_reference_up_to_a_constant():
    o = _ref()
    X, y, _, s2 = O.hlr_synthetic(200, 5, seed=4, has_b=False)
    m = O.HlrModel(X, y, has_b=False, vprior="invgamma")
    rs = np.random.default_rng(1)
    diffs = []
    for _ in range(4):
        theta = rs.standard_normal(5)
        par = np.concatenate([theta, [0.0, s2]])
        ll_ref = O.hlr_ll(o, m, par, list(range(5)))
        ll, _, _ = B.hlr_logp_grad(X, y, theta[None], prior=0, a=s2)
        diffs.append(ll[0] - ll_ref)
    # the theta-dependent part agrees; only the normalising constant differs
    assert np.ptp(diffs) < 1e-9 * max(1.0, abs(diffs[0]))


@pytest.mark.parametrize("prior,a,b", [(0, 2.0, 0.0), (1, 3.0, 1.0), (1, 5.0, 0.5)])
def test_logp_gradient_finite_differences(prior, a, b):
    rs = np.random.default_rng(2)
    X = rs.standard_normal((150, 6))
    y = (rs.random(150) < 0.5).astype(np.int32)
    th = rs.standard_normal((2, 6))
    lp, g, _ = B.hlr_logp_grad(X, y, th, prior, a, b)
    h = 1e-6
    for c in range(2):
        for d in range(6):
            tp, tm = th.copy(), th.copy()
            tp[c, d] += h
            tm[c, d] -= h
            fd = (B.hlr_logp_grad(X, y, tp, prior, a, b)[0][c] - B.hlr_logp_grad(X, y, tm, prior, a, b)[0][c]) / (2 * h)
            assert abs(fd - g[c, d]) < 1e-5 * max(1.0, abs(g[c, d]))


def test_student_t_prior_normalised():
    from scipy import stats
    x = np.linspace(-4, 4, 9)
    ll, _ = B.prior_terms(x[:, None], 1, 3.0, 1.5)
    np.testing.assert_allclose(ll, stats.t.logpdf(x, df=3.0, scale=1.5), rtol=1e-12)


def test_mlp_gradient_finite_differences():
    rs = np.random.default_rng(5)
    din, h1, h2, dout, Bn = 5, 4, 3, 5, 7
    n = h1 * din + h1 + h2 * h1 + h2 + dout * h2 + dout
    w = rs.standard_normal(n) * 0.5
    x = rs.standard_normal((Bn, din))
    t = rs.standard_normal((Bn, dout))
    loss, g = B.mlp_loss_grad(w, w, x, t, din, h1, h2, dout)
    h = 1e-6
    for i in range(n):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (B.mlp_loss_grad(wp, wp, x, t, din, h1, h2, dout)[0] - B.mlp_loss_grad(wm, wm, x, t, din, h1, h2, dout)[0]) / (2 * h)
        assert abs(fd - g[i]) < 1e-6 * max(1.0, abs(g[i]))


def test_ess_of_independent_and_ar1_draws():
    from augurv2_b200.diagnostics import ess
    rs = np.random.default_rng(0)
    x = rs.standard_normal((400, 8, 2))
    e = ess(x)
    assert np.all(e > 0.7 * 3200) and np.all(e < 1.3 * 3200)
    y = np.zeros((3000, 8, 1))
    for t in range(1, 3000):
        y[t] = 0.9 * y[t - 1] + rs.standard_normal((8, 1))
    expect = 3000 * 8 * 0.1 / 1.9
    assert 0.75 * expect < ess(y)[0] < 1.35 * expect
