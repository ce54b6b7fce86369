"""Effective sample size for multi-chain MCMC output.

Multi-chain ESS with Geyer's initial monotone sequence (Geyer 1992; the
chain-combined autocorrelation of Gelman et al., Bayesian Data Analysis,
3rd ed., sec. 11.5):
    rho_t = 1 - (W - mean_c acov_c(t)) / var_plus,
    var_plus = (n - 1) / n * W + B / n,
    tau = -1 + 2 * sum_k P_k,  P_k = rho_2k + rho_2k+1 (positive, monotone),
    ESS = m n / tau.
Host-side post-processing of recorded draws, not part of the sampler.
"""
import numpy as np


def _acov(x):
    """Autocovariance along axis 0 for every column of x [n, k] (biased, FFT)."""
    n = x.shape[0]
    xc = x - x.mean(0, keepdims=True)
    f = np.fft.rfft(xc, n=2 * n, axis=0)
    ac = np.fft.irfft(f * np.conj(f), axis=0)[:n]
    return ac / n


def ess(draws):
    """draws [n_iter, n_chains, n_params] -> ESS per parameter [n_params]."""
    x = np.asarray(draws, dtype=np.float64)
    if x.ndim == 2:
        x = x[:, :, None]
    n, m, k = x.shape
    if n < 4:
        raise ValueError("need at least 4 draws per chain")
    ac = np.stack([_acov(x[:, c, :]) for c in range(m)], axis=1)      # [n, m, k]
    chain_var = ac[0] * n / (n - 1.0)                                   # [m, k]
    W = chain_var.mean(0)
    means = x.mean(0)
    B = n * means.var(0, ddof=1) if m > 1 else np.zeros(k)
    var_plus = (n - 1.0) / n * W + B / n
    var_plus = np.where(var_plus > 0, var_plus, np.finfo(float).tiny)
    rho = 1.0 - (W[None, :] - ac.mean(1)) / var_plus[None, :]          # [n, k]
    rho[0] = 1.0
    out = np.empty(k)
    for j in range(k):
        r = rho[:, j]
        npair = n // 2
        P = r[0:2 * npair:2] + r[1:2 * npair:2]
        tau_sum = 0.0
        prev = np.inf
        for t in range(npair):
            p = P[t]
            if p <= 0:
                break
            p = min(p, prev)
            tau_sum += p
            prev = p
        tau = max(-1.0 + 2.0 * tau_sum, 1.0 / np.log10(max(m * n, 10)))
        out[j] = m * n / tau
    return out
