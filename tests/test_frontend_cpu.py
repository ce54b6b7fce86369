"""The model and schedule languages of the reference parse unchanged, the
supported model families are recognised, and unsupported ones are refused
with NotImplementedError (no silent fallback)."""
import json
import os

import pytest

from augurv2_b200 import augurlib, rv

MODELS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "models.json")))


@pytest.mark.parametrize("name", sorted(MODELS["rv"]))
def test_reference_model_files_parse_and_are_recognised(name):
    m = rv.parse_model(MODELS["rv"][name])
    fam, info = augurlib.recognise(m)
    expect = {"hlr": "hlr", "dethlr": "hlr", "lda": "lda", "mvgmm": "mvgmm", "hmvgmm": "hmvgmm"}[name]
    assert fam == expect
    if name == "dethlr":
        assert info["det"] == "bias"


@pytest.mark.parametrize("ex", sorted(MODELS["examples"]))
def test_example_models_and_schedules_parse(ex):
    rec = MODELS["examples"][ex]
    fam, info = augurlib.recognise(rv.parse_model(rec["model"]))
    for s in rec["scheds"]:
        ks = rv.parse_schedule(s)
        assert ks and all(k.vars for k in ks)
    assert augurlib.default_schedule(fam, info)


def test_schedule_defaults_and_numbers():
    ks = rv.parse_schedule("HMC [theta] (*) NUTS [v, b] [0.1] (*) MWG [v] ~ Normal(v, 1.0) (*) DiscGibbs [z]")
    assert ks[0].params == [1.0, 0.05]          # KernSyn.hs defaults
    assert ks[1].vars == ["v", "b"] and ks[1].params == [0.1]
    assert ks[2].kind == "MWG" and isinstance(ks[2].proposal, rv.Call)
    mwg = rv.parse_schedule("MWG [mu] ~ MvNormal(mu[k], covs0) for k <- 0 until K")[0]
    assert mwg.comps[0].var == "k"


def test_unsupported_model_is_refused():
    src = """(N : Int, lam : Real) => {
      param r ~ Gamma(1.0, lam) ;
      data y[n] ~ Poisson(r) for n <- 0 until N ;
    }"""
    with pytest.raises(NotImplementedError):
        augurlib.recognise(rv.parse_model(src))


def test_glm_regressions_are_recognised():
    """Poisson and linear regressions on dotprod(theta, x[n]) [+ b] with the
    hlr.rv priors run on the HLR engine with their own likelihood; a Normal
    likelihood whose variance is a sampled parameter is refused."""
    pois = """(K : Int, N : Int, lam : Real, x : Vec (Vec Real)) => {
      param v ~ Exponential(lam) ;
      param b ~ Normal(0.0, v) ;
      param theta[k] ~ Normal(0.0, v) for k <- 0 until K ;
      data y[n] ~ Poisson( exp(dotprod(theta, x[n]) + b) ) for n <- 0 until N ;
    }"""
    fam, info = augurlib.recognise(rv.parse_model(pois))
    assert fam == "hlr" and info["lik"] == "poisson" and info["b"] == "b"
    lin = """(K : Int, N : Int, a0 : Real, s0 : Real, s2 : Real, x : Vec (Vec Real)) => {
      param v ~ InvGamma(a0, s0) ;
      param theta[k] ~ Normal(0.0, v) for k <- 0 until K ;
      data y[n] ~ Normal(dotprod(theta, x[n]), s2) for n <- 0 until N ;
    }"""
    fam, info = augurlib.recognise(rv.parse_model(lin))
    assert fam == "hlr" and info["lik"] == "normal" and info["obs_var"].name == "s2" and info["b"] is None
    sampled_var = """(K : Int, N : Int, a0 : Real, s0 : Real, x : Vec (Vec Real)) => {
      param v ~ InvGamma(a0, s0) ;
      param theta[k] ~ Normal(0.0, v) for k <- 0 until K ;
      data y[n] ~ Normal(dotprod(theta, x[n]), v) for n <- 0 until N ;
    }"""
    with pytest.raises(NotImplementedError):
        augurlib.recognise(rv.parse_model(sampled_var))
    no_link = pois.replace("Poisson( exp(dotprod(theta, x[n]) + b) )", "Poisson(dotprod(theta, x[n]) + b)")
    with pytest.raises(NotImplementedError):
        augurlib.recognise(rv.parse_model(no_link))


def test_syntax_errors_are_reported():
    with pytest.raises(rv.RvSyntaxError):
        rv.parse_model("(K : Int) => { param x ~ ; }")
    with pytest.raises(rv.RvSyntaxError):
        rv.parse_schedule("Gibbs [x]")


def test_augur_opt_keeps_reference_signature():
    o = augurlib.AugurOpt(cached=False, target="cpu", paramScale=None)
    assert o.target == "cpu" and o.chains == 1
    with pytest.raises(ValueError):
        augurlib.AugurOpt(target="tpu")
