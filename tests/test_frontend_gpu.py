"""AugurInfer end to end on the GPU with the reference's own example models
and schedules (examples/{lda,hlr,mvgmm}.py), model text unchanged."""
import json
import os

import numpy as np
import pytest

from augurv2_b200.augurdistlib import AugurDefault
from augurv2_b200.augurlib import AugurInfer, AugurOpt
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
MODELS = json.load(open(os.path.join(GOLD, "models.json")))


def test_lda_example_runs_and_matches_direct_sampler():
    g = np.load(os.path.join(GOLD, "lda_d4_k4_v8.npz"))
    off, w = g["doc_off"], g["w"]
    docs = [w[off[d]:off[d + 1]] for d in range(4)]
    N = np.diff(off).astype(np.int32)
    rec = MODELS["examples"]["lda"]
    with AugurInfer("config.yml", rec["model"]) as infer:
        infer.set_compile_opt(AugurOpt(cached=False, target="cpu", paramScale=None, initStrat=AugurDefault()))
        infer.set_user_sched(rec["scheds"][0])
        infer.compile(4, 4, N, g["alpha"], g["beta"])(docs)
        samples = infer.samplen(burnIn=0, numSamples=10)
    # the reference's own run of this fixture (default init, seed 0)
    for it in range(10):
        np.testing.assert_array_equal(np.concatenate(samples["z"][it]), g["z"][it])
        np.testing.assert_allclose(samples["theta"][it], g["theta"][it], rtol=1e-12)


def test_lda_samplen_thinned_pipelined_equals_stepwise():
    """samplen with thin > 1 through the pipelined LDA sample copies equals
    the step-by-step loop (taken when log_like is set), samples and final
    state."""
    g = np.load(os.path.join(GOLD, "lda_d4_k4_v8.npz"))
    off, w = g["doc_off"], g["w"]
    docs = [w[off[d]:off[d + 1]] for d in range(4)]
    N = np.diff(off).astype(np.int32)
    rec = MODELS["examples"]["lda"]
    out = []
    for log_like in (False, True):
        with AugurInfer("config.yml", rec["model"]) as infer:
            infer.set_compile_opt(AugurOpt(cached=False, target="cpu", initStrat=AugurDefault(), seed=3))
            infer.set_user_sched(rec["scheds"][0])
            infer.compile(4, 4, N, g["alpha"], g["beta"])(docs)
            s = infer.samplen(burnIn=2, numSamples=4, thin=3, log_like=log_like)
            out.append((s, infer.backend.get()))
    (sa, fa), (sb, fb) = out
    for name in sa:
        for x, y in zip(sa[name], sb[name]):
            np.testing.assert_array_equal(np.concatenate(x) if name == "z" else x,
                                          np.concatenate(y) if name == "z" else y)
    np.testing.assert_array_equal(np.concatenate(fa["z"]), np.concatenate(fb["z"]))
    np.testing.assert_array_equal(fa["theta"], fb["theta"])


def test_hlr_example_schedules_run():
    rec = MODELS["examples"]["hlr"]
    X, y, beta, s2 = O.hlr_synthetic(500, 6, 3, has_b=True)
    for sched in rec["scheds"]:
        with AugurInfer("config.yml", rec["model"]) as infer:
            infer.set_compile_opt(AugurOpt(cached=False, target="cpu", paramScale=None, seed=1))
            infer.set_user_sched(sched)
            infer.compile(6, 500, 1.0, X)(y)
            s = infer.samplen(burnIn=20, numSamples=30)
            assert len(s["theta"]) == 30 and s["theta"][0].shape == (6,)
            assert np.isfinite(infer.curr_ll())
            assert all(v > 0 for v in s["v"])


def test_hlr_rslice_schedule_runs():
    """The reflective-slice kernel from the schedule language (RSlice [theta]
    [simlen, eps], Rv/ParseRv.y:136) composed with MWG on the variance."""
    rec = MODELS["examples"]["hlr"]
    X, y, beta, s2 = O.hlr_synthetic(500, 6, 3, has_b=True)
    with AugurInfer("config.yml", rec["model"]) as infer:
        infer.set_compile_opt(AugurOpt(cached=False, target="cpu", paramScale=None, seed=2))
        infer.set_user_sched("MWG [v] ~ Normal(v, 0.5) (*) MWG [b] ~ Normal(b, 0.5) (*) RSlice [theta] [0.5, 0.02]")
        infer.compile(6, 500, 1.0, X)(y)
        s = infer.samplen(burnIn=30, numSamples=40)
        th = np.array(s["theta"])
        assert th.shape == (40, 6) and np.isfinite(th).all()
        assert len({tuple(r) for r in th}) > 5, "the reflective slice never moved"
        assert all(v > 0 for v in s["v"])


def test_dethlr_returns_the_deterministic_bias():
    src = MODELS["rv"]["dethlr"]
    X, y, beta, s2 = O.hlr_synthetic(200, 3, 4, has_b=True)
    with AugurInfer(None, src) as infer:
        infer.set_compile_opt(AugurOpt(chains=4, seed=2))
        infer.compile(3, 200, 1.0, X)(y)
        s = infer.samplen(numSamples=3)
        assert s["bias"][0].shape == (4, 200)


@pytest.mark.parametrize("i", [0, 1, 3])
def test_mvgmm_example_schedules_run(i):
    rec = MODELS["examples"]["mvgmm"]
    g = np.load(os.path.join(GOLD, "mvgmm_k3_d2.npz"))
    K, d = 3, 2
    with AugurInfer("config.yml", rec["model"]) as infer:
        infer.set_compile_opt(AugurOpt(cached=False, target="cpu", paramScale=None, seed=3))
        infer.set_user_sched(rec["scheds"][i])
        infer.compile(K, len(g["Y"]), g["mu0"], g["cov0"], g["pis"], g["covs"])(g["Y"])
        s = infer.samplen(numSamples=80)
    mus = np.array(sorted(np.mean(s["mu"][-20:], axis=0).tolist()))
    centres = np.array(sorted([[0.0, 2.0], [2.0, -2.0], [-2.0, -2.0]]))
    assert np.abs(mus - centres).max() < 0.6


def test_hmvgmm_runs_with_default_schedule():
    src = MODELS["rv"]["hmvgmm"]
    Y, z, mus, covs, pis = O.gmm_synthetic(2000, 3, 4, 8)
    with AugurInfer(None, src) as infer:
        infer.set_compile_opt(AugurOpt(seed=4))
        infer.compile(3, 2000, np.ones(3), np.zeros(4), 25 * np.eye(4), 6, np.eye(4))(Y)
        s = infer.samplen(numSamples=10)
    assert s["cov"][-1].shape == (3, 4, 4) and abs(s["pis"][-1].sum() - 1) < 1e-12
