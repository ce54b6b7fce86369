"""The gradient-surrogate network: its device forward/backward against the
FP64 oracle from the same bf16 weights, and what the trained network gains
over the sampler without it."""
import numpy as np
import pytest
import torch

from augurv2_b200 import hlrb as H
from augurv2_b200.diagnostics import ess
from oracle import batched as B

pytestmark = pytest.mark.gpu


def test_mlp_forward_backward_match_fp64():
    D, h1, h2, Bn = 512, 256, 256, 64
    sur = H.MlpSurrogate(D, h1, h2, seed=3)
    gen = torch.Generator("cuda").manual_seed(0)
    x = torch.randn(Bn, D, device="cuda", generator=gen)
    tgt = torch.randn(Bn, D, device="cuda", generator=gen)
    sc = sur._scratch(Bn)
    L = H.N.lib()
    H.N.check(L.ab_mlp_forward(H.C.byref(sur.desc), Bn, H.N.ptr(x), D, H.N.ptr(sc["out"]), D, H.N.ptr(sc["act"]), None))
    H.N.check(L.ab_mlp_mse(Bn, D, H.N.ptr(sc["out"]), D, H.N.ptr(tgt), D, H.N.ptr(sc["dy"]), H.N.ptr(sc["rsq"]), None))
    H.N.check(L.ab_mlp_backward(H.C.byref(sur.desc), Bn, H.N.ptr(x), D, H.N.ptr(sc["dy"]), H.N.ptr(sc["act"]),
                                H.N.ptr(sur.gw), H.N.ptr(sc["bsc"]), None))
    torch.cuda.synchronize()
    wmat = sur.wb.float().double().cpu().numpy()
    wb = sur.w.double().cpu().numpy()
    Y, _ = B.mlp_forward(wmat, wb, x.double().cpu().numpy(), D, h1, h2, D)
    out = sc["out"].double().cpu().numpy()
    assert np.max(np.abs(out - Y)) <= 1e-4 * max(1.0, np.max(np.abs(Y)))
    loss, g = B.mlp_loss_grad(wmat, wb, x.double().cpu().numpy(), tgt.double().cpu().numpy(), D, h1, h2, D)
    gd = sur.gw.double().cpu().numpy()
    # FP32 accumulation against FP64: relative to the largest gradient entry of each block
    n1, n2 = h1 * D, h2 * h1
    offs = [0, n1, n1 + h1, n1 + h1 + n2, n1 + h1 + n2 + h2, n1 + h1 + n2 + h2 + D * h2, len(g)]
    for a, b in zip(offs[:-1], offs[1:]):
        s = np.max(np.abs(g[a:b]))
        assert np.max(np.abs(gd[a:b] - g[a:b])) <= 1e-4 * s, (a, b)
    assert abs(sc["rsq"].sum().item() / (Bn * D) - loss) <= 1e-5 * loss


def test_training_reduces_loss():
    """Adam on the replay buffer lowers the network's error on the part of
    the gradient a per-coordinate linear fit leaves (the dense linear part is
    switched off here so that the network has that part to learn)."""
    D = 64
    sur = H.MlpSurrogate(D, 128, 128, seed=1, batch=256, lr=2e-3, dense_linear=False)
    gen = torch.Generator("cuda").manual_seed(2)
    th = torch.randn(4096, D, device="cuda", generator=gen)
    A = torch.randn(D, D, device="cuda", generator=gen) / D ** 0.5
    g = -th @ A - 0.3 * torch.tanh(th)
    sur.add(th, g)
    sur.refit()
    e0 = sur.rel_error(th[:512], g[:512])
    sur.train(300)
    e1 = sur.rel_error(th[:512], g[:512])
    assert e1 < 0.5 * e0


def _run(sampler, n, record):
    draws = []
    sampler.run(n, record=draws) if record else sampler.run(n)
    return draws


def test_surrogate_gains_over_plain_hmc():
    # N = 100,000 rows, D = 64; 64 chains started at the generating
    # coefficients; both samplers tuned to the same step size.  Cost is
    # counted in exact data passes (a log-density-only pass counts one half
    # of a gradient pass: it is the forward half).
    N_, D, C = 100_000, 64, 64
    X, y, beta = H.synthetic(N_, D, seed=3)
    d = H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0)
    init = np.asarray(beta, np.float32)[None] + 1e-3 * np.random.default_rng(0).standard_normal((C, D)).astype(np.float32)
    eps, L = 0.004, 10
    plain = H.BatchedHmc(d, C, L=L, eps=eps, jitter=0.1, seed=1, init=init)
    plain.run(30)
    plain.reset_stats()
    rec_p = []
    plain.run(120, record=rec_p)
    ess_p = ess(torch.stack(rec_p).cpu().numpy()).min()
    cost_p = 120 * L

    sur = H.SurrogateHmc(d, C, L=L, eps=eps, jitter=0.1, seed=2, init=init, train_every=4, train_steps=40)
    sur.run(60)                        # warm-up: collect pairs and train
    sur.reset_stats()
    g0, l0 = sur.n_grad, sur.n_logp
    rec_s = []
    sur.run(120, record=rec_s)
    ess_s = ess(torch.stack(rec_s).cpu().numpy()).min()
    cost_s = (sur.n_grad - g0) + 0.5 * (sur.n_logp - l0)
    gain = (ess_s / cost_s) / (ess_p / cost_p)
    acc_s = sur.accept_rate()[0]
    print("plain ESS %.1f cost %d acc %s | surrogate ESS %.1f cost %.1f acc %s err %.3f fallback %s gain %.2f" % (
        ess_p, cost_p, plain.accept_rate(), ess_s, cost_s, acc_s, sur.last_rel_err, sur.fallback, gain))
    assert not sur.fallback
    assert gain > 2.0
    assert acc_s > 0.6


@pytest.mark.parametrize("N_,D,factor", [(3000, 16, 0.25), (100_000, 64, 0.75)])
def test_trained_network_gains_over_the_linear_part(N_, D, factor):
    """What the trained network adds to the surrogate's least-squares linear
    part: on fresh exact gradients at the chains' positions after the
    learning warm-up, the relative error of the linear part alone is larger
    by more than 1 / factor (the small-N posterior is the less Gaussian one),
    and the chains accept at least as often with the network as without."""
    C, L = 64, 10
    X, y, beta = H.synthetic(N_, D, seed=5 if N_ < 10_000 else 3)
    d = H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0)
    init = np.asarray(beta, np.float32)[None] + 1e-3 * np.random.default_rng(0).standard_normal((C, D)).astype(np.float32)
    plain = H.BatchedHmc(d, C, L=L, eps=0.01, jitter=0.1, seed=1, init=init)
    eps = H.adapt_step_size(plain, 60)
    sur = H.SurrogateHmc(d, C, L=L, eps=eps, jitter=0.1, seed=2, init=plain.theta.cpu().numpy(), train_every=4,
                         train_steps=40, learn_iters=200)
    sur.run(200)
    assert sur.sur.dense and not sur.fallback
    sur.reset_stats()
    sur.run(80, learn=False)
    acc_net = sur.accept_rate()[0]
    th = sur.theta.clone()
    _, g = d.logp_grad(th)
    e_net = sur.sur.rel_error(th, g)
    sur.sur.use_net = False                 # the same surrogate without its network
    sur._refresh_current()
    e_lin = sur.sur.rel_error(th, g)
    sur.reset_stats()
    sur.run(80, learn=False)
    acc_lin = sur.accept_rate()[0]
    print("N %d D %d: relative error %.4f with the network, %.4f without; accept %.3f / %.3f"
          % (N_, D, e_net, e_lin, acc_net, acc_lin))
    assert e_net < factor * e_lin
    assert acc_net >= acc_lin - 0.02


def test_surrogate_chain_targets_the_exact_posterior():
    # Small HLR (N = 20,000, D = 32, Student-t(3) prior), 256 chains.  The
    # plain GPU sampler's transitions equal the FP64 oracle's
    # (test_hlrb_gpu.test_hmc_transitions_match_fp64_oracle); the surrogate
    # sampler, whose accept test uses the exact log density, must reach the
    # same posterior: every posterior mean within 0.05 posterior sd, and
    # within 5 Monte-Carlo standard errors.
    N_, D, C = 20_000, 32, 256
    X, y, beta = H.synthetic(N_, D, seed=8)
    d = H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0)
    init = np.asarray(beta, np.float32)[None] + 1e-3 * np.random.default_rng(1).standard_normal((C, D)).astype(np.float32)
    plain = H.BatchedHmc(d, C, L=10, eps=0.01, jitter=0.1, seed=21, init=init)
    eps = H.adapt_step_size(plain, 60)
    plain.run(100)
    start = plain.theta.cpu().numpy()
    plain.capture()
    rec_p = []
    plain.run(400, record=rec_p)
    sur = H.SurrogateHmc(d, C, L=10, eps=eps, jitter=0.1, seed=22, init=start, train_every=4, train_steps=10)
    sur.run(100)
    sur.capture()
    rec_s = []
    sur.run(400, record=rec_s)
    dp = torch.stack(rec_p).cpu().numpy()
    ds = torch.stack(rec_s).cpu().numpy()
    ep, es = ess(dp), ess(ds)
    mp, ms = dp.reshape(-1, D).mean(0), ds.reshape(-1, D).mean(0)
    sd = dp.reshape(-1, D).std(0)
    z = (ms - mp) / (sd * np.sqrt(1.0 / ep + 1.0 / es))
    print("min ESS plain %.0f surrogate %.0f; max |diff|/sd %.4f; max |z| %.2f; accept %s %s" % (
        ep.min(), es.min(), np.max(np.abs(ms - mp) / sd), np.max(np.abs(z)), plain.accept_rate(), sur.accept_rate()))
    assert np.max(np.abs(ms - mp) / sd) < 0.05
    assert np.max(np.abs(z)) < 5.0
    sd_s = ds.reshape(-1, D).std(0)
    assert np.all(np.abs(sd_s / sd - 1.0) < 0.1)


def test_nan_surrogate_falls_back_to_exact_hmc():
    """Host-side fault injection: the network's weights are overwritten with
    NaN mid-run.  Trajectories it drives are rejected by the exact log
    density (the chains stay finite), the next error check measures a NaN
    error and switches the sampler to exact-gradient HMC, which accepts
    again; no GPU fault is involved."""
    N_, D, C = 20_000, 16, 32
    X, y, beta = H.synthetic(N_, D, seed=6)
    d = H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0)
    init = np.asarray(beta, np.float32)[None] + 1e-3 * np.random.default_rng(0).standard_normal((C, D)).astype(np.float32)
    sur = H.SurrogateHmc(d, C, L=5, eps=0.01, jitter=0.1, seed=2, init=init, train_every=4, train_steps=5)
    sur.run(8)
    assert not sur.fallback
    before = sur.theta.clone()
    sur.sur.w.fill_(float("nan"))
    sur.sur.a.fill_(float("nan"))
    N_check = 4 - sur.it % 4
    sur.run(N_check)                      # up to and including the next check
    assert sur.fallback and not np.isfinite(sur.last_rel_err)
    assert torch.isfinite(sur.theta).all()
    sur.reset_stats()
    sur.run(12)                           # exact-gradient HMC from here
    assert torch.isfinite(sur.theta).all()
    assert sur.accept_rate()[0] > 0.3
    assert not torch.equal(before, sur.theta)
