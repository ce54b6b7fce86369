"""Scalar conjugate Gibbs updates on the GPU: host side of ab_conj_scalar.

The reference library carries seven one-parameter conjugate pairs
(cbits/augur_dist.c:185-195, 314-336, 408-412) that its compiler never
emits (its conjugacy detector knows Dirichlet-Categorical, MvNormal-MvNormal
and InvWishart-MvNormal only, compiler/augur/src/Core/CgConj.hs:313-342).
`ScalarConj` runs any of them as one batched step over G groups, for
hierarchical models whose group g has a scalar parameter with a conjugate
prior and ragged observations x[g][0 .. n_g):

    kind                prior on the group's parameter   observations
    beta_bernoulli      Beta(h0, h1)                      Bernoulli(p)
    beta_geometric      Beta(h0, h1)                      Geometric(p) (failures)
    gamma_poisson       Gamma(h0, rate h1)                Poisson(l)
    gamma_exponential   Gamma(h0, rate h1)                Exponential(rate l)
    gamma_gammashape    Gamma(h0, rate h1)                Gamma(a_n, rate b)
    gamma_invgamma      Gamma(h0, rate h1)                InvGamma(a_n, scale b)
    normal_normalmean   Normal(h0, var h1)                Normal(m, var h2)

The observations stay on the device; each `step` forms the statistics and
draws every group's parameter in one launch (conj.cu), from Philox
substream (group, iteration, 15), so a run is reproducible and the CPU
oracle reproduces it to rounding.
"""
import numpy as np
import torch

from . import _native as N
from .checkpoint import Checkpointable

KINDS = {
    "beta_bernoulli": 0,
    "beta_geometric": 1,
    "gamma_poisson": 2,
    "gamma_exponential": 3,
    "gamma_gammashape": 4,
    "gamma_invgamma": 5,
    "normal_normalmean": 6,
}
SHAPED = ("gamma_gammashape", "gamma_invgamma")


def _groups(x):
    """Ragged groups (sequence of 1-D arrays) or (offsets, flat) -> CSR."""
    if isinstance(x, tuple) and len(x) == 2:
        off = np.ascontiguousarray(x[0], dtype=np.int64)
        flat = np.ascontiguousarray(x[1], dtype=np.float64).ravel()
    else:
        rows = [np.asarray(r, dtype=np.float64).ravel() for r in x]
        off = np.zeros(len(rows) + 1, dtype=np.int64)
        np.cumsum([len(r) for r in rows], out=off[1:])
        flat = np.concatenate(rows) if rows else np.zeros(0)
    if off[0] != 0 or np.any(np.diff(off) < 0) or off[-1] != len(flat):
        raise ValueError("group offsets must start at 0, be nondecreasing and end at the data length")
    if off[-1] >= 2**31:
        raise ValueError("more than 2^31 observations")
    return off.astype(np.int32), flat


class ScalarConj(Checkpointable):
    """G conjugate scalar parameters updated together.

    x: ragged observations per group (list of arrays, or (offsets, flat));
    aux: the observations' known shapes (same layout) for gamma_gammashape /
    gamma_invgamma; h0, h1, h2: prior hyper-parameters (and the known
    observation variance h2 of normal_normalmean), scalars or arrays of G.
    """
    _ckpt_tensors = ("value",)
    _ckpt_scalars = ("iteration", "seed")

    def __init__(self, kind, x, h0, h1, h2=None, aux=None, seed=0, iter0=0, device="cuda"):
        if kind not in KINDS:
            raise ValueError("kind must be one of %s" % ", ".join(KINDS))
        self.kind, self.code = kind, KINDS[kind]
        self.dev = torch.device(device)
        off, flat = _groups(x)
        self.G = len(off) - 1
        if kind in SHAPED:
            if aux is None:
                raise ValueError("%s needs aux (the observations' known shapes)" % kind)
            aoff, aflat = _groups(aux)
            if not np.array_equal(aoff, off):
                raise ValueError("aux must have the observations' layout")
            self.aux = torch.as_tensor(aflat, device=self.dev)
        else:
            self.aux = None
        if kind == "normal_normalmean" and h2 is None:
            raise ValueError("normal_normalmean needs h2 (the observation variance)")
        per = [np.ndim(h) > 0 for h in (h0, h1, h2) if h is not None]
        self.per_group = int(any(per))
        hs = []
        for h in (h0, h1, h2 if h2 is not None else 0.0):
            a = np.asarray(h, dtype=np.float64)
            a = np.broadcast_to(a, (self.G,)) if self.per_group else a.reshape(1)
            hs.append(torch.tensor(np.array(a, dtype=np.float64), device=self.dev))
        self.h0, self.h1, self.h2 = hs
        self.off = torch.as_tensor(off, device=self.dev)
        self.x = torch.as_tensor(flat, device=self.dev)
        self.value = torch.full((self.G,), float("nan"), dtype=torch.float64, device=self.dev)
        self.stat_sum = torch.zeros(self.G, dtype=torch.float64, device=self.dev)
        self.stat_aux = torch.zeros(self.G, dtype=torch.float64, device=self.dev)
        self.seed, self.iteration = int(seed), int(iter0)

    def step(self, n=1, stream=None):
        """n Gibbs updates of every group's parameter (the statistics do not
        depend on the parameter, so each update is one independent draw from
        the group's posterior)."""
        L = N.lib()
        st = N.stream_ptr(stream)
        for _ in range(int(n)):
            N.check(L.ab_conj_scalar(self.code, self.G, N.ptr(self.off), N.ptr(self.x), N.ptr(self.aux),
                                     N.ptr(self.h0), N.ptr(self.h1), N.ptr(self.h2), self.per_group,
                                     N.ptr(self.stat_sum), N.ptr(self.stat_aux), N.ptr(self.value),
                                     self.seed, self.iteration, st), "ab_conj_scalar")
            self.iteration += 1
        return self.value

    def stats(self):
        """(sum, aux sum or count) per group, from the last step."""
        return self.stat_sum.cpu().numpy(), self.stat_aux.cpu().numpy()

    def get(self):
        return self.value.cpu().numpy()
