"""Bindings from a recognised model (augurlib.recognise) and its schedule to
the GPU samplers.  Each backend replaces what the reference's generated
library does behind augur_iface_init / augur_step / augur_cpy /
augur_set_pt / augur_get_curr_ll (compiler/augur/src/CudaC/CgStInit.hs:
474-602, CgKern.hs:232-238): it uploads the data once, steps the sampler
on the device, and copies samples back into numpy values shaped like the
reference's (nested vectors become lists / arrays)."""
import numpy as np

from . import rv
from .augurdistlib import AugurDefault, AugurRandom, AugurUser, init_value


class Unsupported(NotImplementedError):
    pass


def _val(e, hyp):
    return rv.const_value(e, hyp)


def _names_by_role(info, role_map):
    return {info[r]: r for r in role_map if info.get(r)}


# ---------------------------------------------------------------------------
class LdaBackend:
    def __init__(self, info, parsed, sched, hyp, data, opt):
        from .lda import LdaGibbs, flatten_docs
        kinds = [(k.kind, k.vars) for k in sched]
        want = {("ConjGibbs", (info["theta"],)), ("ConjGibbs", (info["phi"],)), ("DiscGibbs", (info["z"],))}
        if len(kinds) != 3 or {(k, tuple(v)) for k, v in kinds} != want or kinds[2][0] != "DiscGibbs":
            raise Unsupported("LDA runs ConjGibbs on %s and %s, then DiscGibbs [%s]"
                              % (info["theta"], info["phi"], info["z"]))
        self.info = info
        alpha = np.asarray(hyp[info["alpha"]], np.float64)
        beta = np.asarray(hyp[info["beta"]], np.float64)
        K, V = len(alpha), len(beta)
        docs = data[0]
        off, w = flatten_docs(docs)
        D = len(off) - 1
        self.doc_off, self.w, self.alpha, self.beta = off, w, alpha, beta
        rng = np.random.default_rng(opt.seed)
        strat = opt.initStrat
        if isinstance(strat, AugurUser):
            theta = np.asarray(strat.initPt[info["theta"]], np.float64)
            phi = np.asarray(strat.initPt[info["phi"]], np.float64)
            z = np.concatenate([np.asarray(x, np.int32) for x in strat.initPt[info["z"]]])
        else:
            theta = np.array([init_value(strat, "Dirichlet", [alpha], rng) for _ in range(D)])
            phi = np.array([init_value(strat, "Dirichlet", [beta], rng) for _ in range(K)])
            z = np.zeros(len(w), np.int32)
            if isinstance(strat, AugurRandom):
                for d in range(D):
                    for t in range(off[d], off[d + 1]):
                        z[t] = init_value(strat, "Categorical", [theta[d]], rng)
        self.s = LdaGibbs(K, V, off, w, alpha, beta, seed=opt.seed, theta=theta, phi=phi, z=z, device=opt.device)
        self.param_names = [info["theta"], info["phi"], info["z"]]

    def step(self, n):
        self.s.sweep(n)

    def get(self):
        theta, phi, z = self.s.state()
        off = self.doc_off
        return {self.info["theta"]: theta, self.info["phi"]: phi,
                self.info["z"]: [z[off[d]:off[d + 1]] for d in range(len(off) - 1)]}

    def samples(self, n, first, every):
        """get() after `first` steps and then every `every` steps, n times,
        with each copy to the host overlapping the next steps."""
        off = self.doc_off
        for theta, phi, z in self.s.samples(n, first, every):
            yield {self.info["theta"]: theta, self.info["phi"]: phi,
                   self.info["z"]: [z[off[d]:off[d + 1]] for d in range(len(off) - 1)]}

    def set_pt(self, pt):
        z = np.concatenate([np.asarray(x, np.int32) for x in pt[self.info["z"]]])
        self.s.set_state(theta=pt[self.info["theta"]], phi=pt[self.info["phi"]], z=z)

    def state_dict(self):
        return self.s.state_dict()

    def load_state_dict(self, d):
        self.s.load_state_dict(d)

    def curr_ll(self):
        """Joint log density in the reference's terms (augur_get_curr_ll,
        CgStInit.hs:597-602; augur_dirichlet_ll has no normalising constant,
        cbits/augur_dist.c:488-496), on the device."""
        return self.s.ll_mod()


# ---------------------------------------------------------------------------
class HlrBackend:
    def __init__(self, info, parsed, sched, hyp, data, opt):
        from .hlr import HlrChains, HlrData
        self.info = info
        X = np.asarray(hyp[info["x"]], np.float64)
        if X.dtype == object:
            X = np.array([np.asarray(r, np.float64) for r in X])
        lik = info.get("lik", "bernoulli")
        y = np.asarray(data[0], np.float64 if lik == "normal" else np.int32)
        obs_var = float(_val(info["obs_var"], hyp)) if lik == "normal" else 1.0
        vp = info["vprior"]
        if vp.fn == "Exponential":
            pri = dict(vprior="exponential", lam=_val(vp.args[0], hyp))
        else:
            pri = dict(vprior="invgamma", a0=_val(vp.args[0], hyp), s0=_val(vp.args[1], hyp))
        self.has_b = info["b"] is not None
        self.X = X
        self.data = HlrData(X, y, has_b=self.has_b, compat=opt.compat, x_dtype=opt.x_dtype,
                            device=opt.device, lik=lik, obs_var=obs_var, **pri)
        role = {info["theta"]: "theta", info["v"]: "v"}
        if self.has_b:
            role[info["b"]] = "b"
        comps = []
        for k in sched:
            for v in k.vars:
                if v not in role:
                    raise Unsupported("%s is not a sampled parameter of this model" % v)
            if k.kind == "HMC":
                comps.append({"kind": "HMC", "block": [role[v] for v in k.vars], "simlen": k.params[0],
                              "eps": k.params[1]})
            elif k.kind == "NUTS":
                comps.append({"kind": "NUTS", "block": [role[v] for v in k.vars], "eps": k.params[0],
                              "max_depth": opt.max_depth})
            elif k.kind == "RSlice":
                comps.append({"kind": "RSlice", "block": [role[v] for v in k.vars], "simlen": k.params[0],
                              "eps": k.params[1]})
            elif k.kind == "MWG":
                p = k.proposal
                v = k.vars[0]
                if not (isinstance(p, rv.Call) and p.fn == "Normal" and isinstance(p.args[0], rv.Var)
                        and p.args[0].name == v and role[v] != "theta"):
                    raise Unsupported("MWG supports scalar Normal(x, s) random-walk proposals")
                comps.append({"kind": "MWG", "var": role[v], "scale": _val(p.args[1], hyp)})
            else:
                raise Unsupported("%s is not available for this model on the B200 backend" % k.kind)
        D = X.shape[1]
        C = opt.chains
        rng = np.random.default_rng(opt.seed)
        init = np.zeros((C, D + 2))
        strat = opt.initStrat
        for c in range(C):
            if isinstance(strat, AugurUser):
                pt = strat.initPt
                v = float(pt[info["v"]])
                init[c, :D] = np.asarray(pt[info["theta"]], np.float64)
                init[c, D] = float(pt[info["b"]]) if self.has_b else 0.0
            else:
                vargs = [_val(a, hyp) for a in vp.args]
                v = init_value(strat, vp.fn, vargs, rng)
                init[c, :D] = [init_value(strat, "Normal", [0.0, v], rng) for _ in range(D)]
                init[c, D] = init_value(strat, "Normal", [0.0, v], rng) if self.has_b else 0.0
            init[c, D + 1] = v
        self.D, self.C = D, C
        self.chains = HlrChains(self.data, comps, C=C, init=init, seed=opt.seed)
        self.param_names = [n for n in info["order"]] + ([info["det"]] if info["det"] else [])

    def step(self, n):
        self.chains.run(n)

    def get(self):
        s = self.chains.state()
        D = self.D
        out = {}
        pick = (lambda a: a[0]) if self.C == 1 else (lambda a: a)
        out[self.info["theta"]] = pick(s[:, :D].copy())
        out[self.info["v"]] = pick(s[:, D + 1].copy())
        if self.has_b:
            out[self.info["b"]] = pick(s[:, D].copy())
        if self.info["det"]:
            out[self.info["det"]] = pick(self.chains.det_bias().cpu().numpy())
        if self.C == 1:
            for k in (self.info["v"], self.info["b"]):
                if k in out:
                    out[k] = float(out[k])
        return out

    def set_pt(self, pt):
        import torch
        D = self.D
        s = self.chains.state()
        s[:, :D] = np.asarray(pt[self.info["theta"]], np.float64)
        s[:, D + 1] = np.asarray(pt[self.info["v"]], np.float64)
        if self.has_b:
            s[:, D] = np.asarray(pt[self.info["b"]], np.float64)
        self.chains.pars.copy_(torch.as_tensor(s))

    def state_dict(self):
        return self.chains.state_dict()

    def load_state_dict(self, d):
        self.chains.load_state_dict(d)

    def curr_ll(self):
        """Joint log density (augur_get_curr_ll, CgStInit.hs:597-602): the
        block of all parameters has every factor in its full conditional."""
        from .hlr import block_indices, ll_grad
        names = ["v"] + (["b"] if self.has_b else []) + ["theta"]
        ll, _ = ll_grad(self.data, self.chains.state(), block_indices(names, self.D))
        return float(ll[0]) if self.C == 1 else ll


# ---------------------------------------------------------------------------
class GmmBackend:
    def __init__(self, family, info, parsed, sched, hyp, data, opt):
        from .gmm import GmmGibbs
        self.info, self.family = info, family
        Y = np.asarray(data[0], np.float64)
        Y = np.array([np.asarray(r, np.float64).ravel() for r in Y]) if Y.dtype == object else Y.reshape(len(Y), -1)
        mu0 = np.asarray(hyp[info["mu0"]], np.float64).ravel()
        cov0 = np.asarray(hyp[info["cov0"]], np.float64)
        d = Y.shape[1]
        K = None
        mu_decl = parsed.decl(info["mu"])
        if mu_decl.comps:
            K = int(_val(mu_decl.comps[0].hi, hyp))
        rng = np.random.default_rng(opt.seed)
        strat = opt.initStrat
        kinds = [k.kind for k in sched]
        if family == "mvgmm":
            if len(sched) != 2 or sched[1].kind != "DiscGibbs" or sched[0].kind not in ("ConjGibbs", "ESlice", "MWG"):
                raise Unsupported("mvgmm runs ConjGibbs, ESlice or MWG on %s, then DiscGibbs [%s]"
                                  % (info["mu"], info["z"]))
            move = {"ConjGibbs": "conj", "ESlice": "eslice", "MWG": "mwg"}[sched[0].kind]
            prop_cov = None
            if move == "mwg":
                p = sched[0].proposal
                if not (isinstance(p, rv.Call) and p.fn == "MvNormal" and isinstance(p.args[1], rv.Var)):
                    raise Unsupported("MWG [mu] ~ MvNormal(mu[k], S) with S a hyper-parameter")
                prop_cov = np.asarray(hyp[p.args[1].name], np.float64)
            pis = np.asarray(hyp[info["pis"]], np.float64)
            covs = np.asarray(hyp[info["covs"]], np.float64)
            mu, z = self._init_mu_z(strat, K, mu0, cov0, pis, len(Y), rng)
            self.s = GmmGibbs(Y, K, mu0, cov0, pis=pis, covs=covs, mu=mu, z=z, move=move, prop_cov=prop_cov,
                              compat=opt.compat, seed=opt.seed, device=opt.device)
        else:
            want = ["ConjGibbs"] * 3 + ["DiscGibbs"]
            if kinds != want or [k.vars[0] for k in sched] != [info["pis"], info["mu"], info["cov"], info["z"]]:
                raise Unsupported("hmvgmm runs ConjGibbs [%s] (*) ConjGibbs [%s] (*) ConjGibbs [%s] (*) DiscGibbs [%s]"
                                  % (info["pis"], info["mu"], info["cov"], info["z"]))
            alpha = np.asarray(hyp[info["alpha"]], np.float64)
            df = int(_val(info["df"], hyp))
            scale0 = np.asarray(hyp[info["scale0"]], np.float64)
            K = len(alpha) if K is None else K
            if isinstance(strat, AugurUser):
                pis = np.asarray(strat.initPt[info["pis"]], np.float64)
                cov = np.asarray(strat.initPt[info["cov"]], np.float64)
            else:
                pis = init_value(strat, "Dirichlet", [alpha], rng)
                cov = np.array([init_value(strat, "InvWishart", [df, scale0], rng) for _ in range(K)])
            mu, z = self._init_mu_z(strat, K, mu0, cov0, pis, len(Y), rng)
            self.s = GmmGibbs(Y, K, mu0, cov0, alpha=alpha, df=df, scale0=scale0, pis=pis, mu=mu, cov=cov, z=z,
                              seed=opt.seed, device=opt.device)
        self.K, self.Y = K, Y
        self.param_names = list(info["order"])

    def _init_mu_z(self, strat, K, mu0, cov0, pis, N, rng):
        if isinstance(strat, AugurUser):
            return (np.asarray(strat.initPt[self.info["mu"]], np.float64),
                    np.asarray(strat.initPt[self.info["z"]], np.int32))
        mu = np.array([init_value(strat, "MvNormal", [mu0, cov0], rng) for _ in range(K)])
        z = np.array([init_value(strat, "Categorical", [pis], rng) for _ in range(N)], np.int32)
        return mu, z

    def step(self, n):
        self.s.sweep(n)

    def get(self):
        st = self.s.state()
        out = {self.info["mu"]: st["mu"], self.info["z"]: st["z"]}
        if self.family == "hmvgmm":
            out[self.info["pis"]] = st["pis"]
            out[self.info["cov"]] = st["cov"]
        return out

    def set_pt(self, pt):
        kw = {"mu": pt[self.info["mu"]], "z": pt[self.info["z"]]}
        if self.family == "hmvgmm":
            kw.update(pis=pt[self.info["pis"]], cov=pt[self.info["cov"]])
        self.s.set_state(**kw)

    def state_dict(self):
        return self.s.state_dict()

    def load_state_dict(self, d):
        self.s.load_state_dict(d)

    def curr_ll(self):
        """Joint log density in the reference's terms (augur_get_curr_ll,
        CgStInit.hs:597-602), on the device."""
        return self.s.ll_mod()


def make(family, info, parsed, sched, hyp, data, opt):
    if family == "lda":
        return LdaBackend(info, parsed, sched, hyp, data, opt)
    if family == "hlr":
        return HlrBackend(info, parsed, sched, hyp, data, opt)
    return GmmBackend(family, info, parsed, sched, hyp, data, opt)
