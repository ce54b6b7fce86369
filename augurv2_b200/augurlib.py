"""AugurInfer / AugurOpt - the reference's Python front end
(pyaugur/pyaugur/augurlib.py:34-222) on the B200 backend.

A model and schedule written for the reference run unchanged:

    with AugurInfer('config.yml', augur_lda) as infer:
        infer.set_compile_opt(AugurOpt(cached=False, target='cpu'))
        infer.set_user_sched('ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z]')
        infer.compile(K, D, N, alpha, beta)(w)
        samples = infer.samplen(burnIn=0, numSamples=100)

Instead of compiling the model to C/CUDA (hs_compile, augurlib.py:263-308)
and a per-model library (augurlib.py:310-423), the model text is parsed
(rv.py), recognised as one of the model families that the CUDA library
implements, and bound to its sampler: LDA (lda.rv), hierarchical logistic
regression (hlr.rv, dethlr.rv and the InvGamma-variance variant), Gaussian
mixtures with shared covariance (mvgmm.rv) and with per-component
covariances and weights (hmvgmm.rv).  Any other model raises
NotImplementedError.  Every target ('cpu', 'gpu', 'b200') runs on the GPU;
there is no CPU path.

Extra options go in AugurOpt keyword arguments: chains (independent chains,
one thread block each for HLR), seed, compat (the reference's own density
formulas), x_dtype ('f32' | 'bf16' storage of the design matrix),
max_depth (NUTS), device.
"""
import math
import os

import numpy as np

from . import rv

try:  # the reference's init strategies, reproduced for API compatibility
    from .augurdistlib import AugurDefault, AugurInitStrat, AugurRandom, AugurUser  # noqa: F401
except ImportError:  # pragma: no cover
    raise


class AugurOpt:
    """Compile options (augurlib.py:34-48), plus B200 options as keywords."""

    def __init__(self, cached=False, target="cpu", initStrat=None, paramScale=None, chains=1, seed=0,
                 compat=True, x_dtype="f32", max_depth=10, device="cuda"):
        if target not in ("cpu", "gpu", "b200"):
            raise ValueError("target must be 'cpu', 'gpu' or 'b200'")
        self.cached, self.target = cached, target
        self.initStrat = initStrat if initStrat is not None else AugurRandom()
        if not isinstance(self.initStrat, AugurInitStrat):
            raise TypeError("initStrat must be an AugurInitStrat")
        self.paramScale = paramScale
        self.chains, self.seed, self.compat = int(chains), int(seed), bool(compat)
        self.x_dtype, self.max_depth, self.device = x_dtype, int(max_depth), device


def logmsg(s):
    print(s)


# ---- model recognition -------------------------------------------------------------
class Unsupported(NotImplementedError):
    pass


def _is_var(e, name=None):
    return isinstance(e, rv.Var) and (name is None or e.name == name)


def _is_idx(e, base=None, n=None):
    return (isinstance(e, rv.Index) and _is_var(e.base, base)
            and (n is None or len(e.idx) == n))


def _hyper_kinds(model):
    return dict(model.hparams)


def recognise(model):
    """Returns (family, info) for a supported model, else raises Unsupported."""
    params = [d for d in model.decls if d.kind == "param" and d.dist is not None]
    dets = [d for d in model.decls if d.kind == "param" and d.dist is None]
    datas = [d for d in model.decls if d.kind == "data"]
    if len(datas) != 1:
        raise Unsupported("models with exactly one data declaration are supported")
    y = datas[0]
    fn = y.dist.fn
    if fn in ("Bernoulli", "Poisson", "Normal"):
        return "hlr", _rec_hlr(model, params, dets, y)
    if fn == "Categorical":
        return "lda", _rec_lda(model, params, dets, y)
    if fn == "MvNormal":
        return _rec_gmm(model, params, dets, y)
    raise Unsupported("no B200 sampler for a %s likelihood" % fn)


def _rec_hlr(model, params, dets, y):
    """Regressions on a linear predictor t = dotprod(theta, x[n]) [+ b] with
    theta[k] ~ Normal(0, v), b ~ Normal(0, v), v ~ Exponential | InvGamma:
    y[n] ~ Bernoulli(sigmoid(t)) (hlr.rv, dethlr.rv), Poisson(exp(t)) or
    Normal(t, s2) with s2 a hyper-parameter or a number."""
    fn = y.dist.fn
    arg = y.dist.args[0]
    det = None
    if _is_idx(arg) and len(dets) == 1 and arg.base.name == dets[0].name:
        det = dets[0]
        arg = det.expr
    elif dets:
        raise Unsupported("deterministic declarations other than the bias of hlr")
    obs_var = None
    if fn == "Bernoulli":
        if not (isinstance(arg, rv.Call) and arg.fn == "sigmoid"):
            raise Unsupported("Bernoulli(sigmoid(...)) expected")
        lin = arg.args[0]
    elif fn == "Poisson":
        if det is not None or not (isinstance(arg, rv.Call) and arg.fn == "exp"):
            raise Unsupported("Poisson(exp(...)) expected")
        lin = arg.args[0]
    else:
        if det is not None or len(y.dist.args) != 2:
            raise Unsupported("Normal(dotprod(theta, x[n]) [+ b], s2) expected")
        lin, obs_var = arg, y.dist.args[1]
        if _is_var(obs_var) and obs_var.name in {d.name for d in params}:
            raise Unsupported("the observation variance of a Normal likelihood must be a hyper-parameter")
    bias = None
    if isinstance(lin, rv.BinOp) and lin.op == "+":
        lin, bias = lin.lhs, lin.rhs
        if not _is_var(bias):
            raise Unsupported("bias must be a parameter")
    if not (isinstance(lin, rv.Call) and lin.fn == "dotprod" and len(lin.args) == 2):
        raise Unsupported("sigmoid(dotprod(theta, x[n]) [+ b]) expected")
    th, xn = lin.args
    if not (_is_var(th) and _is_idx(xn, n=1)):
        raise Unsupported("dotprod(theta, x[n]) expected")
    byname = {d.name: d for d in params}
    theta = byname.get(th.name)
    if theta is None or theta.dist.fn != "Normal" or len(theta.idxs) != 1:
        raise Unsupported("theta[k] ~ Normal(0.0, v) expected")
    vname = theta.dist.args[1].name if _is_var(theta.dist.args[1]) else None
    v = byname.get(vname)
    if v is None or v.dist.fn not in ("Exponential", "InvGamma"):
        raise Unsupported("the variance must have an Exponential or InvGamma prior")
    names = {theta.name, v.name}
    b = None
    if bias is not None:
        b = byname.get(bias.name)
        if b is None or b.dist.fn != "Normal" or not _is_var(b.dist.args[1], v.name):
            raise Unsupported("b ~ Normal(0.0, v) expected")
        names.add(b.name)
    if set(byname) != names:
        raise Unsupported("unexpected parameters %s" % sorted(set(byname) - names))
    return {"theta": theta.name, "b": b.name if b else None, "v": v.name, "x": xn.base.name,
            "y": y.name, "vprior": v.dist, "det": det.name if det else None, "order": [d.name for d in params],
            "lik": {"Bernoulli": "bernoulli", "Poisson": "poisson", "Normal": "normal"}[fn], "obs_var": obs_var}


def _rec_lda(model, params, dets, w):
    if dets or len(params) != 3 or len(w.idxs) != 2:
        raise Unsupported("LDA expects theta, phi, z and w[d, n]")
    z = next((d for d in params if d.dist.fn == "Categorical"), None)
    if z is None or len(z.idxs) != 2:
        raise Unsupported("z[d, n] ~ Categorical(theta[d]) expected")
    th_e = z.dist.args[0]
    ph_e = w.dist.args[0]
    if not (_is_idx(th_e, n=1) and _is_idx(ph_e, n=1) and _is_idx(ph_e.idx[0], z.name, 2)):
        raise Unsupported("w[d, n] ~ Categorical(phi[z[d, n]]) expected")
    byname = {d.name: d for d in params}
    theta, phi = byname.get(th_e.base.name), byname.get(ph_e.base.name)
    if theta is None or phi is None or theta.dist.fn != "Dirichlet" or phi.dist.fn != "Dirichlet":
        raise Unsupported("Dirichlet priors on theta and phi expected")
    nlen = w.comps[1].hi
    return {"theta": theta.name, "phi": phi.name, "z": z.name, "w": w.name,
            "alpha": theta.dist.args[0].name, "beta": phi.dist.args[0].name,
            "K": phi.comps[0].hi.name if phi.comps else None, "D": theta.comps[0].hi.name if theta.comps else None,
            "N": nlen.base.name if _is_idx(nlen) else None}


def _rec_gmm(model, params, dets, y):
    if dets:
        raise Unsupported("deterministic declarations are not supported for mixtures")
    mean_e, cov_e = y.dist.args
    byname = {d.name: d for d in params}
    if not (_is_idx(mean_e, n=1) and _is_idx(mean_e.idx[0], n=1)):
        raise Unsupported("y[n] ~ MvNormal(mu[z[n]], ...) expected")
    mu = byname.get(mean_e.base.name)
    z = byname.get(mean_e.idx[0].base.name)
    if mu is None or z is None or mu.dist.fn != "MvNormal" or z.dist.fn != "Categorical":
        raise Unsupported("mu[k] ~ MvNormal and z[n] ~ Categorical expected")
    info = {"mu": mu.name, "z": z.name, "y": y.name, "mu0": mu.dist.args[0].name, "cov0": mu.dist.args[1].name,
            "order": [d.name for d in params]}
    pis_e = z.dist.args[0]
    if _is_var(cov_e):                       # mvgmm: shared covariance hyper, fixed weights
        if set(byname) != {mu.name, z.name} or not _is_var(pis_e):
            raise Unsupported("mvgmm expects mu and z only")
        info.update(covs=cov_e.name, pis=pis_e.name)
        return "mvgmm", info
    if not (_is_idx(cov_e, n=1) and _is_idx(cov_e.idx[0], z.name, 1)):
        raise Unsupported("y[n] ~ MvNormal(mu[z[n]], cov[z[n]]) expected")
    cov = byname.get(cov_e.base.name)
    pis = byname.get(pis_e.name) if _is_var(pis_e) else None
    if cov is None or cov.dist.fn != "InvWishart" or pis is None or pis.dist.fn != "Dirichlet":
        raise Unsupported("hmvgmm expects pis ~ Dirichlet and cov[k] ~ InvWishart")
    info.update(cov=cov.name, pis=pis.name, alpha=pis.dist.args[0].name, df=cov.dist.args[0],
                scale0=cov.dist.args[1].name)
    return "hmvgmm", info


def default_schedule(family, info):
    """kernHeuristic1 (compiler/augur/src/Compile/Compile.hs:143-166): per
    parameter in model order, ConjGibbs when conjugate, DiscGibbs when
    discrete, otherwise HMC [v] with simLen 1.0, eps 0.05."""
    if family == "lda":
        return "ConjGibbs [%s] (*) ConjGibbs [%s] (*) DiscGibbs [%s]" % (info["theta"], info["phi"], info["z"])
    if family == "mvgmm":
        return "ConjGibbs [%s] (*) DiscGibbs [%s]" % (info["mu"], info["z"])
    if family == "hmvgmm":
        return "ConjGibbs [%s] (*) ConjGibbs [%s] (*) ConjGibbs [%s] (*) DiscGibbs [%s]" % (
            info["pis"], info["mu"], info["cov"], info["z"])
    return " (*) ".join("HMC [%s]" % p for p in info["order"])


# ---- the front end -------------------------------------------------------------------
class AugurInfer:
    def __init__(self, path_config=None, model=None):
        if model is None and path_config is not None and not os.path.exists(str(path_config)):
            path_config, model = None, path_config
        self.model = model
        self.config = {}
        if path_config is not None and os.path.exists(path_config):
            import yaml
            with open(path_config) as f:
                self.config = yaml.safe_load(f) or {}
        self.aopt = None
        self.userSched = None
        self.backend = None
        self.param_names = []

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_value, traceback):
        self.backend = None

    # ---- public interface (augurlib.py:146-222) --------------------------------------
    def set_compile_opt(self, aopt):
        self.aopt = aopt
        return self

    def set_user_sched(self, userSched):
        self.userSched = userSched
        return self

    def compile(self, *hypers):
        def _compile(*data):
            if self.aopt is None:
                raise NameError("Set compiler options first...")
            parsed = rv.parse_model(self.model)
            family, info = recognise(parsed)
            sched = rv.parse_schedule(self.userSched or default_schedule(family, info))
            hyp = {name: val for (name, _), val in zip(parsed.hparams, hypers)}
            if len(hypers) != len(parsed.hparams):
                raise ValueError("model takes %d hyper-parameters, got %d" % (len(parsed.hparams), len(hypers)))
            from . import backends
            self.backend = backends.make(family, info, parsed, sched, hyp, data, self.aopt)
            self.param_names = self.backend.param_names
        return _compile

    def curr_ll(self):
        assert self.backend is not None
        return self.backend.curr_ll()

    def checkpoint(self, path):
        """Save the sampler's state (device tensors, iteration counters) to
        `path`; resume() on a model compiled with the same data continues the
        chains bit for bit (no reference counterpart: the reference keeps its
        state in process globals)."""
        import torch
        assert self.backend is not None
        torch.save({"param_names": list(self.param_names), "state": self.backend.state_dict()}, path)

    def resume(self, path):
        import torch
        assert self.backend is not None
        d = torch.load(path, weights_only=False)
        if list(d["param_names"]) != list(self.param_names):
            raise ValueError("checkpoint of a model with parameters %s, this one has %s"
                             % (d["param_names"], self.param_names))
        self.backend.load_state_dict(d["state"])

    def sample(self):
        assert self.backend is not None
        self.backend.step(1)
        return self.backend.get()

    def samplen(self, burnIn=0, numSamples=1, thin=1, log_like=False):
        assert self.backend is not None
        if burnIn:
            self.backend.step(burnIn)
        samples = {name: [] for name in self.param_names}
        # a sample after the first step and then after every `thin` steps
        # (augurlib.py:207-221)
        if not log_like and numSamples > 0 and hasattr(self.backend, "samples"):
            # the same samples, each copied out while the next steps run
            for cur in self.backend.samples(numSamples, 1, thin):
                for name in self.param_names:
                    samples[name].append(cur[name])
            if thin > 1:
                self.backend.step(thin - 1)
            return samples
        pending = 0
        for i in range(numSamples * thin):
            pending += 1
            if i % thin == 0:
                self.backend.step(pending)
                pending = 0
                cur = self.backend.get()
                if log_like:
                    print("log-like[%d]: %f" % (i // thin, self.curr_ll()))
                for name in self.param_names:
                    samples[name].append(cur[name])
        if pending:
            self.backend.step(pending)
        return samples

    def set_pt(self, pt):
        for p in self.param_names:
            assert p in pt
        self.backend.set_pt(pt)
