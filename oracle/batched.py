"""ORACLE (test infrastructure only): FP64 restatements for the batched HLR
path, the batched HMC transition and the gradient-surrogate network.

* hlr_logp_grad - the HLR block log density and gradient of the reference's
  generated code (CgLike.hs:139-147 over augur_bernoulli_ll, augur_dist.c:
  59-66; CgGrad.hs:345-376 with augur_bernoulli_dotarg1 x augur_expit_grad_0,
  augur_dist.c:68-71, augur_math.c:56-59) for many chains at once, with the
  Normal(0, var) prior (augur_normal_ll, augur_dist.c:372-381, written with
  the correct density here) or a Student-t prior;
* hmc_iteration - one transition of h_augur_mcmc_hmc / h_augur_mcmc_leapfrog
  (cbits/augur_mcmclib.h:343-424) per chain, fed the same Philox draws as the
  device driver (momenta: tag MOM, one normal per coordinate; jitter and
  accept uniforms: tag HMC positions 0 and 1);
* mlp_* - forward, mean-squared-error loss and backward of the d-h1-h2-d GELU
  network in FP64 from the same (bf16-rounded) weights.
Only tests/ and bench.py's CPU baseline use this module.
"""
import math

import numpy as np
from scipy.special import erf, gammaln

TAG_MOM, TAG_HMC = 4, 5


def prior_terms(theta, prior, a, b):
    th = np.asarray(theta, np.float64)
    if prior == 0:
        ll = -0.5 * np.log(2.0 * np.pi * a) - 0.5 * th * th / a
        g = -th / a
    else:
        nu, z = a, th / b
        ll = (gammaln(0.5 * (nu + 1.0)) - gammaln(0.5 * nu) - 0.5 * np.log(nu * np.pi) - np.log(b)
              - 0.5 * (nu + 1.0) * np.log1p(z * z / nu))
        g = -(nu + 1.0) * th / (nu * b * b + th * th)
    return ll.sum(-1), g


def hlr_logp_grad(X, y, theta, prior=1, a=3.0, b=1.0):
    """X [N, D] (float64 values of the bf16 data), y [N], theta [C, D] ->
    logp [C], grad [C, D], and the per-coordinate scale sum_n |r x| used to
    state gradient tolerances."""
    X = np.asarray(X, np.float64)
    th = np.asarray(theta, np.float64)
    yv = np.asarray(y, np.float64)
    t = th @ X.T                                        # [C, N]
    sp = np.logaddexp(0.0, t)                           # softplus
    ll = (yv * t - sp).sum(-1)
    r = yv - 1.0 / (1.0 + np.exp(-t))
    g = r @ X
    scale = np.abs(r) @ np.abs(X)
    pl, pg = prior_terms(th, prior, a, b)
    return ll + pl, g + pg, scale


def hmc_iteration(o, X, y, theta, g_cur, logp_cur, eps0, jitter, L, seed, it, prior=1, a=3.0, b=1.0):
    """One HMC transition for every chain (FP64).  o is an oracle.Oracle for
    the Philox draws.  Returns (theta, g, logp, accepted[C], dH[C])."""
    th = np.array(theta, np.float64)
    g = np.array(g_cur, np.float64)
    lp = np.array(logp_cur, np.float64)
    C_, D = th.shape
    out_th, out_g, out_lp = th.copy(), g.copy(), lp.copy()
    acc = np.zeros(C_, bool)
    dHs = np.zeros(C_)
    for c in range(C_):
        hu = o.draws(seed, c, it, TAG_HMC, 2)
        eps = eps0 * (1.0 + jitter * (2.0 * hu[0] - 1.0))
        p = o.draws(seed, c, it, TAG_MOM, D, normal=True)
        H0 = -lp[c] + 0.5 * np.dot(p, p)
        x = th[c].copy()
        p = p + 0.5 * eps * g[c]
        x = x + eps * p
        for l in range(L):
            lpn, gn, _ = hlr_logp_grad(X, y, x[None], prior, a, b)
            if l < L - 1:
                p = p + eps * gn[0]
                x = x + eps * p
        p = p + 0.5 * eps * gn[0]
        H1 = -lpn[0] + 0.5 * np.dot(p, p)
        dH = H0 - H1
        dHs[c] = dH
        if np.isfinite(H1) and math.log(hu[1]) < dH:
            acc[c] = True
            out_th[c], out_g[c], out_lp[c] = x, gn[0], lpn[0]
    return out_th, out_g, out_lp, acc, dHs


def _gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def _gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def mlp_unpack(w, d_in, h1, h2, d_out):
    w = np.asarray(w, np.float64)
    k = 0
    out = []
    for (r, c) in ((h1, d_in), (h2, h1), (d_out, h2)):
        out.append(w[k:k + r * c].reshape(r, c)); k += r * c
        out.append(w[k:k + r]); k += r
    return out


def mlp_forward(w_mat, w_bias, x, d_in, h1, h2, d_out):
    """Weights from w_mat (bf16-rounded master), biases from w_bias (master)."""
    W1, _, W2, _, W3, _ = mlp_unpack(w_mat, d_in, h1, h2, d_out)
    _, b1, _, b2, _, b3 = mlp_unpack(w_bias, d_in, h1, h2, d_out)
    x = np.asarray(x, np.float64)
    P1 = x @ W1.T + b1
    A1 = _gelu(P1)
    P2 = A1 @ W2.T + b2
    A2 = _gelu(P2)
    Y = A2 @ W3.T + b3
    return Y, (P1, A1, P2, A2)


def mlp_loss_grad(w_mat, w_bias, x, target, d_in, h1, h2, d_out):
    """Mean squared error and its gradient (flat parameter layout)."""
    W1, _, W2, _, W3, _ = mlp_unpack(w_mat, d_in, h1, h2, d_out)
    Y, (P1, A1, P2, A2) = mlp_forward(w_mat, w_bias, x, d_in, h1, h2, d_out)
    B = Y.shape[0]
    E = Y - np.asarray(target, np.float64)
    loss = (E * E).sum() / (B * d_out)
    dY = 2.0 * E / (B * d_out)
    dW3 = dY.T @ A2
    db3 = dY.sum(0)
    dP2 = (dY @ W3) * _gelu_grad(P2)
    dW2 = dP2.T @ A1
    db2 = dP2.sum(0)
    dP1 = (dP2 @ W2) * _gelu_grad(P1)
    dW1 = dP1.T @ np.asarray(x, np.float64)
    db1 = dP1.sum(0)
    grad = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, grad
