"""Hierarchical logistic regression on the GPU: host side of ab_hlr_*.

Model (compiler/augur/test/hlr.rv):
    v ~ Exponential(lam)            (or InvGamma(a0, s0))
    b ~ Normal(0, v)                (optional)
    theta[k] ~ Normal(0, v)         for k < D
    y[n] ~ Bernoulli(sigmoid(dotprod(theta, x[n]) + b))
or, with the same priors, y[n] ~ Poisson(exp(dotprod(theta, x[n]) + b)) or
y[n] ~ Normal(dotprod(theta, x[n]) + b, obs_var) (lik="poisson" / "normal").
A chain's parameters are one f64 vector [theta[0..D-1], b, v]; schedule
components (HMC / NUTS / MWG) move blocks of it.  All chains run on the
device, one thread block per chain (hlr.cu).
"""
import ctypes as C

import numpy as np
import torch

from . import _native as N
from .checkpoint import Checkpointable
from .trace import traced

HMC, NUTS, MWG, RSLICE = 0, 1, 2, 3


class HlrComp(C.Structure):
    _fields_ = [("kind", C.c_int), ("P", C.c_int), ("idx_off", C.c_int), ("max_depth", C.c_int),
                ("simlen", C.c_double), ("eps", C.c_double), ("mwg_var", C.c_double)]


class HlrModelC(C.Structure):
    _fields_ = [("N", C.c_int), ("D", C.c_int), ("ldx", C.c_int), ("has_b", C.c_int),
                ("vprior", C.c_int), ("compat", C.c_int), ("x_dtype", C.c_int),
                ("lam", C.c_double), ("a0", C.c_double), ("s0", C.c_double),
                ("X", C.c_void_p), ("y", C.c_void_p), ("lik", C.c_int), ("obs_var", C.c_double),
                ("yr", C.c_void_p)]


LIKELIHOODS = {"bernoulli": 0, "poisson": 1, "normal": 2}


def block_indices(names, D):
    """Schedule block (list of 'theta', 'b', 'v') -> indices into par."""
    out = []
    for n in names:
        if n == "theta":
            out += list(range(D))
        elif n == "b":
            out.append(D)
        elif n == "v":
            out.append(D + 1)
        else:
            raise ValueError("unknown HLR parameter %r" % n)
    return out


class HlrData:
    """Design matrix and labels resident on the device (f32 or bf16).
    lik: "bernoulli" (0/1 labels), "poisson" (counts) or "normal" (real
    labels, observation variance obs_var)."""

    def __init__(self, X, y, has_b=True, vprior="exponential", lam=1.0, a0=1.0, s0=1.0,
                 compat=True, x_dtype="f32", device="cuda", lik="bernoulli", obs_var=1.0):
        X = np.asarray(X)
        self.N, self.D = X.shape
        tdt = {"f32": torch.float32, "bf16": torch.bfloat16}[x_dtype]
        self.X = torch.as_tensor(np.ascontiguousarray(X, dtype=np.float32)).to(device=device, dtype=tdt)
        self.lik = LIKELIHOODS[lik]
        self.obs_var = float(obs_var)
        if self.lik == LIKELIHOODS["normal"]:
            self.yr = torch.as_tensor(np.ascontiguousarray(y, dtype=np.float32)).to(device)
            self.y = torch.zeros(self.N, dtype=torch.int32, device=device)
        else:
            self.y = torch.as_tensor(np.ascontiguousarray(y, dtype=np.int32)).to(device)
            self.yr = None
        self.has_b = bool(has_b)
        self.vprior = {"exponential": 0, "invgamma": 1}[vprior]
        self.compat = bool(compat)
        self.x_dtype = {"f32": 0, "bf16": 1}[x_dtype]
        self.lam, self.a0, self.s0 = float(lam), float(a0), float(s0)
        self.c = HlrModelC(self.N, self.D, self.D, int(self.has_b), self.vprior, int(self.compat),
                           self.x_dtype, self.lam, self.a0, self.s0, self.X.data_ptr(), self.y.data_ptr(),
                           self.lik, self.obs_var, self.yr.data_ptr() if self.yr is not None else None)


def ll_grad(data, pars, idx, stream=None):
    """Block log full-conditional and gradient for each row of pars [C, D+2]."""
    pars_t = torch.as_tensor(np.ascontiguousarray(pars, np.float64)).to(data.X.device)
    C_ = pars_t.shape[0]
    idx_h = np.ascontiguousarray(idx, np.int32)
    idx_d = torch.as_tensor(idx_h).to(data.X.device)
    ll = torch.zeros(C_, dtype=torch.float64, device=data.X.device)
    g = torch.zeros((C_, len(idx_h)), dtype=torch.float64, device=data.X.device)
    N.check(N.lib().ab_hlr_ll_grad(C.byref(data.c), N.ptr(idx_d), idx_h.ctypes.data_as(C.c_void_p),
                                   len(idx_h), C_, N.ptr(pars_t), N.ptr(ll), N.ptr(g),
                                   N.stream_ptr(stream)), "ab_hlr_ll_grad")
    return ll.cpu().numpy(), g.cpu().numpy()


class HlrChains(Checkpointable):
    _ckpt_tensors = ("pars", "stats")
    _ckpt_scalars = ("iteration", "seed")

    """C chains of a schedule over one HLR data set.

    schedule: list of dicts, e.g.
      {"kind": "HMC", "block": ["theta"], "simlen": 0.5, "eps": 0.05}
      {"kind": "NUTS", "block": ["v", "b", "theta"], "eps": 0.05, "max_depth": 10}
      {"kind": "MWG", "var": "v", "scale": 1.0}
      {"kind": "RSlice", "block": ["theta"], "simlen": 1.0, "eps": 0.05}
    """

    def __init__(self, data, schedule, C=1, init=None, seed=0, iter0=0):
        self.data, self.C, self.seed, self.iteration = data, int(C), int(seed), int(iter0)
        D = data.D
        comps, idx = [], []
        for s in schedule:
            kind = s["kind"].upper()
            if kind == "MWG":
                bl = block_indices([s["var"]], D)
                comps.append(HlrComp(MWG, 1, len(idx), 0, 0.0, 0.0, float(s.get("scale", 1.0))))
            else:
                bl = block_indices(s["block"], D)
                if kind == "HMC":
                    comps.append(HlrComp(HMC, len(bl), len(idx), 0, float(s.get("simlen", 1.0)),
                                         float(s.get("eps", 0.05)), 0.0))
                elif kind == "NUTS":
                    comps.append(HlrComp(NUTS, len(bl), len(idx), int(s.get("max_depth", 10)), 0.0,
                                         float(s.get("eps", 0.05)), 0.0))
                elif kind == "RSLICE":
                    comps.append(HlrComp(RSLICE, len(bl), len(idx), 0, float(s.get("simlen", 1.0)),
                                         float(s.get("eps", 0.05)), 0.0))
                else:
                    raise ValueError("unknown component kind %r" % s["kind"])
            idx += bl
        self.ncomp = len(comps)
        self.comps_h = (HlrComp * len(comps))(*comps)
        dev = data.X.device
        self.comps_d = torch.as_tensor(np.frombuffer(bytes(self.comps_h), dtype=np.uint8).copy()).to(dev)
        self.idx_h = np.ascontiguousarray(idx, np.int32)
        self.idx_d = torch.as_tensor(self.idx_h).to(dev)
        if init is None:
            init = np.zeros((self.C, D + 2))
            init[:, D + 1] = 1.0
        init = np.broadcast_to(np.asarray(init, np.float64), (self.C, D + 2)).copy()
        self.pars = torch.as_tensor(np.ascontiguousarray(init)).to(dev)
        # per chain and component: accepts, NUTS depth, NUTS leaves / RSlice
        # reflections, stack overflows, divergent iterations
        self.stats = torch.zeros((self.C, self.ncomp, 5), dtype=torch.float64, device=dev)
        need_nuts = any(c.kind == NUTS for c in comps)
        nbytes = int(N.lib().ab_hlr_chain_scratch_bytes(self.C, D)) if need_nuts else 8
        self.scratch = torch.zeros(nbytes, dtype=torch.uint8, device=dev)

    def det_bias(self, stream=None):
        """dethlr.rv's deterministic bias[n] = sigmoid(dotprod(theta, x[n]) + b)
        of every chain, [C, N] float64, computed on the device."""
        out = torch.empty((self.C, self.data.N), dtype=torch.float64, device=self.pars.device)
        N.check(N.lib().ab_hlr_det(C.byref(self.data.c), self.C, N.ptr(self.pars), N.ptr(out),
                                   N.stream_ptr(stream)), "ab_hlr_det")
        return out

    def divergences(self):
        """Divergent HMC / NUTS iterations per component, summed over chains."""
        return self.stats[:, :, 4].sum(0).cpu().numpy()

    @traced("hlr.run_chains")
    def run(self, n_iter=1, stream=None):
        N.check(N.lib().ab_hlr_run_chains(C.byref(self.data.c), self.comps_h, N.ptr(self.comps_d),
                                          self.ncomp, N.ptr(self.idx_d),
                                          self.idx_h.ctypes.data_as(C.c_void_p), self.C, N.ptr(self.pars),
                                          int(n_iter), self.iteration, self.seed, N.ptr(self.stats),
                                          N.ptr(self.scratch), N.stream_ptr(stream)), "ab_hlr_run_chains")
        self.iteration += int(n_iter)

    def state(self):
        return self.pars.cpu().numpy()
