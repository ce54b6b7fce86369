"""Checkpoint / resume on the GPU: a sampler restored from a checkpoint
continues bit for bit as the uninterrupted run (counter-based Philox draws,
state fully in device tensors), through the pyaugur-style front end
(AugurInfer.checkpoint / resume) and for the batched samplers."""
import json
import os

import numpy as np
import pytest
import torch

from augurv2_b200 import hlrb as H
from augurv2_b200.augurlib import AugurInfer, AugurOpt
from augurv2_b200.lda import synthetic_corpus
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
MODELS = json.load(open(os.path.join(GOLD, "models.json")))


def _equal(a, b):
    assert a.keys() == b.keys()
    for k in a:
        x, y = a[k], b[k]
        if isinstance(x, list):
            for u, v in zip(x, y):
                np.testing.assert_array_equal(np.asarray(u), np.asarray(v))
        else:
            np.testing.assert_array_equal(np.asarray(x), np.asarray(y))


def _resume_matches(make, n1, n2, path):
    """make() -> compiled AugurInfer.  Uninterrupted n1 + n2 steps against
    n1 steps, checkpoint, a fresh compile, resume, n2 steps."""
    a = make()
    a.samplen(numSamples=n1 + n2)
    want = a.backend.get()
    b = make()
    b.samplen(numSamples=n1)
    b.checkpoint(path)
    c = make()
    c.resume(path)
    c.samplen(numSamples=n2)
    _equal(want, c.backend.get())


def test_lda_resume(tmp_path):
    rec = MODELS["examples"]["lda"]
    off, w = synthetic_corpus(6, 80, 12, 30, 0.1, 0.01, seed=3)
    docs = [w[off[d]:off[d + 1]] for d in range(12)]

    def make():
        inf = AugurInfer("config.yml", rec["model"])
        inf.set_compile_opt(AugurOpt(cached=False, target="cpu", seed=4))
        inf.set_user_sched(rec["scheds"][0])
        inf.compile(6, 12, [len(x) for x in docs], np.full(6, 0.1), np.full(80, 0.01))(docs)
        return inf
    _resume_matches(make, 5, 7, str(tmp_path / "lda.pt"))


def test_hlr_resume(tmp_path):
    rec = MODELS["examples"]["hlr"]
    X, y, beta, s2 = O.hlr_synthetic(300, 5, 2, has_b=True)

    def make():
        inf = AugurInfer("config.yml", rec["model"])
        inf.set_compile_opt(AugurOpt(cached=False, target="cpu", seed=6, chains=4))
        inf.set_user_sched(rec["scheds"][1])
        inf.compile(5, 300, 1.0, X)(y)
        return inf
    _resume_matches(make, 6, 5, str(tmp_path / "hlr.pt"))


def test_hmvgmm_resume(tmp_path):
    src = MODELS["rv"]["hmvgmm"]
    Y, z, mus, covs, pis = O.gmm_synthetic(600, 3, 4, 7)

    def make():
        inf = AugurInfer(None, src)
        inf.set_compile_opt(AugurOpt(seed=8))
        inf.compile(3, 600, np.ones(3), np.zeros(4), 25 * np.eye(4), 6, np.eye(4))(Y)
        return inf
    _resume_matches(make, 4, 4, str(tmp_path / "gmm.pt"))


def _hlrb_data(N, D, seed):
    rs = np.random.default_rng(seed)
    X = torch.as_tensor(rs.standard_normal((N, D)), dtype=torch.float32).to(torch.bfloat16)
    beta = rs.standard_normal(D) * 0.3
    y = (rs.random(N) < 1 / (1 + np.exp(-(X.double().numpy() @ beta)))).astype(np.int32)
    return H.HlrbData(X, y, prior="normal", var=2.0), beta


def test_batched_hmc_and_nuts_resume(tmp_path):
    d, beta = _hlrb_data(3000, 16, 1)
    init = (beta[None] + 0.01 * np.random.default_rng(2).standard_normal((8, 16))).astype(np.float32)
    a = H.BatchedHmc(d, 8, L=4, eps=0.02, seed=3, init=init)
    a.run(6)
    b = H.BatchedHmc(d, 8, L=4, eps=0.02, seed=3, init=init)
    b.run(3)
    b.save(str(tmp_path / "hmc.pt"))
    c = H.BatchedHmc(d, 8, L=4, eps=0.02, seed=3, init=np.zeros((8, 16), np.float32))
    c.load(str(tmp_path / "hmc.pt"))
    c.run(3)
    assert torch.equal(a.theta, c.theta) and torch.equal(a.s.stats, c.s.stats)

    a = H.BatchedNuts(d, 8, eps=0.02, max_depth=6, seed=5, init=init, hist_cap=64)
    a.run(120)
    b = H.BatchedNuts(d, 8, eps=0.02, max_depth=6, seed=5, init=init, hist_cap=64)
    b.run(50)
    b.save(str(tmp_path / "nuts.pt"))
    c = H.BatchedNuts(d, 8, eps=0.02, max_depth=6, seed=5, init=init, hist_cap=64)
    c.load(str(tmp_path / "nuts.pt"))
    c.capture()                                   # a resumed sampler can capture its round
    c.run(69)                                     # capture ran one round itself
    np.testing.assert_array_equal(a.draws(), c.draws())
    np.testing.assert_array_equal(a.info(), c.info())


def test_surrogate_hmc_resume(tmp_path):
    d, beta = _hlrb_data(4000, 32, 4)
    init = (beta[None] + 1e-3 * np.random.default_rng(1).standard_normal((16, 32))).astype(np.float32)

    def make():
        return H.SurrogateHmc(d, 16, L=5, eps=0.01, seed=9, init=init, train_every=4, train_steps=3)
    a = make()
    a.run(12)
    b = make()
    b.run(6)
    b.save(str(tmp_path / "sur.pt"))
    c = make()
    c.load(str(tmp_path / "sur.pt"))
    c.run(6)
    assert torch.equal(a.theta, c.theta)
    assert (a.it, a.fallback, a.n_grad, a.n_logp) == (c.it, c.fallback, c.n_grad, c.n_logp)
    assert torch.equal(a.sur.w, c.sur.w)
