"""ORACLE (test infrastructure only).

ctypes front end of the two CPU checkers:

* ``Oracle("oracle")`` - the standalone C restatement (oracle/augur_oracle.c,
  built into oracle/_build/liboracle.so);
* ``Oracle("ref")`` - the reference's own cbits runtime compiled in place with
  the GSL shim and the restated generated code (oracle/_ref/libaugur_ref.so).

Both export the same functions under the prefixes ``orc_`` and ``ref_``; this
module hides the prefix so a test can run the same call on both and compare.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {
    "oracle": os.path.join(HERE, "_build", "liboracle.so"),
    "ref": os.path.join(HERE, "_ref", "libaugur_ref.so"),
}
PREFIX = {"oracle": "orc_", "ref": "ref_"}

TAG_Z, TAG_THETA, TAG_PHI, TAG_MOM, TAG_HMC, TAG_NUTS = 1, 2, 3, 4, 5, 6
TAG_PI, TAG_MU, TAG_COV, TAG_ESLICE, TAG_MWG, TAG_INIT, TAG_DATA = 7, 8, 9, 10, 11, 12, 13
TAG_RSLICE, TAG_CONJ = 14, 15

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u32p = C.POINTER(C.c_uint32)


# The reference checkout sits beside this repository unless REF_SRC names
# its cbits directory.
REF_SRC_DEFAULT = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "cbits")


def build_oracle():
    """Compile the standalone oracle (and the reference build when the
    reference sources are present) with oracle/Makefile."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    ref_src = os.environ.get("REF_SRC", REF_SRC_DEFAULT)
    if os.path.isdir(ref_src):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", "REF_SRC=" + os.path.abspath(ref_src)])


def available(kind):
    return os.path.exists(LIBS[kind])


def dptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


class Oracle:
    def __init__(self, kind="oracle"):
        path = LIBS[kind]
        if not os.path.exists(path):
            if kind == "oracle":
                build_oracle()
            else:
                raise FileNotFoundError(path)
        self.kind = kind
        self.lib = C.CDLL(path)
        self.p = PREFIX[kind]

    def fn(self, name, restype=None):
        f = getattr(self.lib, self.p + name)
        f.restype = restype
        return f

    # ---- scalar samplers --------------------------------------------------
    def gamma_sample(self, shape, rate, seed, elem, it, tag):
        f = self.fn("gamma_sample", C.c_double)
        f.argtypes = [C.c_double, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        return f(shape, rate, seed, elem, it, tag)

    def unnorm_disc_samp(self, pmf, seed, elem, it, tag):
        pmf = np.ascontiguousarray(pmf, dtype=np.float64)
        f = self.fn("unnorm_disc_samp", C.c_int)
        f.argtypes = [_dp, C.c_int, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        return f(dptr(pmf), len(pmf), seed, elem, it, tag)

    def philox_block(self, ctr, key):
        ctr = np.asarray(ctr, dtype=np.uint32)
        out = np.zeros(4, dtype=np.uint32)
        f = self.fn("philox_block")
        f(ctr.ctypes.data_as(_u32p), C.c_uint32(key[0]), C.c_uint32(key[1]), out.ctypes.data_as(_u32p))
        return out

    def draws(self, seed, elem, it, tag, n, normal=False):
        out = np.zeros(n, dtype=np.float64)
        f = self.fn("draws")
        f.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int, _dp]
        f(seed, elem, it, tag, n, int(normal), dptr(out))
        return out

    # ---- scalar conjugate updates ----------------------------------------------
    def conj_scalar(self, kind, off, x, h0, h1, h2=None, aux=None, seed=0, it=0):
        """Per-group statistics and draws; returns (out, stat_sum, stat_aux).
        h0 / h1 / h2: scalars or arrays of G values."""
        off = np.ascontiguousarray(off, dtype=np.int32)
        G = len(off) - 1
        x = np.ascontiguousarray(x, dtype=np.float64)
        aux = None if aux is None else np.ascontiguousarray(aux, dtype=np.float64)
        per_group = int(np.ndim(h0) > 0)
        hs = [np.ascontiguousarray(np.atleast_1d(h if h is not None else 0.0), dtype=np.float64)
              for h in (h0, h1, h2)]
        out, ssum, saux = (np.zeros(G) for _ in range(3))
        f = self.fn("conj_scalar")
        f.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp,
                      C.c_uint64, C.c_uint32]
        f(kind, G, iptr(off), dptr(x) if len(x) else None, dptr(aux) if aux is not None and len(aux) else None,
          dptr(hs[0]), dptr(hs[1]), dptr(hs[2]), per_group, dptr(ssum), dptr(saux), dptr(out), seed, it)
        return out, ssum, saux

    # ---- LDA ----------------------------------------------------------------
    def lda_disc_z(self, doc_off, w, theta, phi, z, seed, it):
        D, K = theta.shape
        V = phi.shape[1]
        f = self.fn("lda_disc_z")
        f.argtypes = [C.c_int] * 3 + [_ip, _ip, _dp, _dp, _ip, C.c_uint64, C.c_uint32]
        f(D, K, V, iptr(doc_off), iptr(w), dptr(theta), dptr(phi), iptr(z), seed, it)
        return z

    def lda_conj_stat(self, doc_off, w, z, D, K, V):
        cnt_dk = np.zeros((D, K), np.int32)
        cnt_kw = np.zeros((K, V), np.int32)
        f = self.fn("lda_conj_stat")
        f.argtypes = [C.c_int] * 3 + [_ip, _ip, _ip, _ip, _ip]
        f(D, K, V, iptr(doc_off), iptr(w), iptr(z), iptr(cnt_dk), iptr(cnt_kw))
        return cnt_dk, cnt_kw

    def lda_conj_theta(self, alpha, cnt_dk, seed, it):
        D, K = cnt_dk.shape
        out = np.zeros((D, K), np.float64)
        f = self.fn("lda_conj_theta")
        f.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp, C.c_uint64, C.c_uint32]
        f(D, K, dptr(alpha), iptr(cnt_dk), dptr(out), seed, it)
        return out

    def lda_conj_phi(self, beta, cnt_kw, seed, it):
        K, V = cnt_kw.shape
        out = np.zeros((K, V), np.float64)
        f = self.fn("lda_conj_phi")
        f.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp, C.c_uint64, C.c_uint32]
        f(K, V, dptr(beta), iptr(cnt_kw), dptr(out), seed, it)
        return out

    def lda_ll_mod(self, doc_off, w, z, alpha, beta, theta, phi):
        """The model log density augur_get_curr_ll returns for lda.rv."""
        D, K = theta.shape
        V = phi.shape[1]
        f = self.fn("lda_ll_mod", C.c_double)
        f.argtypes = [C.c_int] * 3 + [_ip, _ip, _ip, _dp, _dp, _dp, _dp]
        c = np.ascontiguousarray
        return f(D, K, V, iptr(c(doc_off, np.int32)), iptr(c(w, np.int32)), iptr(c(z, np.int32)),
                 dptr(c(alpha, np.float64)), dptr(c(beta, np.float64)), dptr(c(theta, np.float64)),
                 dptr(c(phi, np.float64)))

    def lda_pred_ll(self, doc_off, w, theta, phi):
        """Held-out log-likelihood of one theta sample (oracle only)."""
        D, K = theta.shape
        V = phi.shape[1]
        f = self.fn("lda_pred_ll", C.c_double)
        f.argtypes = [C.c_int] * 3 + [_ip, _ip, _dp, _dp]
        c = np.ascontiguousarray
        return f(D, K, V, iptr(c(doc_off, np.int32)), iptr(c(w, np.int32)), dptr(c(theta, np.float64)),
                 dptr(c(phi, np.float64)))

    def lda_sweeps(self, doc_off, w, alpha, beta, theta, phi, z, seed, it0, n):
        D, K = theta.shape
        V = phi.shape[1]
        cnt_dk = np.zeros((D, K), np.int32)
        cnt_kw = np.zeros((K, V), np.int32)
        f = self.fn("lda_sweeps")
        f.argtypes = [C.c_int] * 3 + [_ip, _ip, _dp, _dp, _dp, _dp, _ip, _ip, _ip,
                                      C.c_uint64, C.c_uint32, C.c_int]
        f(D, K, V, iptr(doc_off), iptr(w), dptr(alpha), dptr(beta), dptr(theta), dptr(phi),
          iptr(z), iptr(cnt_dk), iptr(cnt_kw), seed, it0, n)
        return theta, phi, z


# ---- HLR -------------------------------------------------------------------
class OrcHlr(C.Structure):
    _fields_ = [("N", C.c_int), ("D", C.c_int), ("has_b", C.c_int), ("vprior", C.c_int),
                ("compat", C.c_int), ("lam", C.c_double), ("a0", C.c_double), ("s0", C.c_double),
                ("X", _dp), ("y", _ip), ("lik", C.c_int), ("obs_var", C.c_double), ("yr", _dp)]


LIKELIHOODS = {"bernoulli": 0, "poisson": 1, "normal": 2}


class HlrModel:
    """Data and hyper-parameters of one HLR instance (oracle side).
    vprior: "exponential" (hlr.rv, rate lam) or "invgamma" (a0, s0).
    lik: "bernoulli" (y ~ Bernoulli(sigmoid(t))), "poisson" (y ~
    Poisson(exp(t))) or "normal" (y ~ Normal(t, obs_var), y real), with
    t = theta . x[n] + b."""

    def __init__(self, X, y, has_b=True, vprior="exponential", lam=1.0, a0=1.0, s0=1.0, compat=True,
                 lik="bernoulli", obs_var=1.0):
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.lik = LIKELIHOODS[lik]
        if self.lik == 2:
            self.yr = np.ascontiguousarray(y, dtype=np.float64)
            self.y = np.zeros(len(self.yr), np.int32)
        else:
            self.y = np.ascontiguousarray(y, dtype=np.int32)
            self.yr = np.zeros(len(self.y), np.float64)
        self.obs_var = float(obs_var)
        self.N, self.D = self.X.shape
        self.has_b, self.compat = int(has_b), int(compat)
        self.vprior = {"exponential": 0, "invgamma": 1}[vprior]
        self.lam, self.a0, self.s0 = float(lam), float(a0), float(s0)

    def struct(self):
        return OrcHlr(self.N, self.D, self.has_b, self.vprior, self.compat, self.lam, self.a0, self.s0,
                      dptr(self.X), iptr(self.y), self.lik, self.obs_var, dptr(self.yr))

    def flat(self):
        return (self.N, self.D, self.has_b, self.vprior, self.lam, self.a0, self.s0,
                dptr(self.X), iptr(self.y))


_FLAT = [C.c_int] * 4 + [C.c_double] * 3 + [_dp, _ip]


def _hlr_call(o, name, m, restype, extra_types, *extra):
    f = o.fn(name, restype)
    if o.kind == "ref":
        if not m.compat:
            raise ValueError("the reference build only has the reference's own densities")
        g = o.fn("glm_set", None)
        g.argtypes = [C.c_int, C.c_double, _dp]
        g(m.lik, m.obs_var, dptr(m.yr))
        f.argtypes = _FLAT + extra_types
        return f(*m.flat(), *extra)
    s = m.struct()
    f.argtypes = [C.POINTER(OrcHlr)] + extra_types
    return f(C.byref(s), *extra)


def _idx(idx):
    return np.ascontiguousarray(idx, dtype=np.int32)


def hlr_ll(o, m, par, idx):
    par = np.ascontiguousarray(par, np.float64); idx = _idx(idx)
    return _hlr_call(o, "hlr_ll", m, C.c_double, [_dp, _ip, C.c_int], dptr(par), iptr(idx), len(idx))


def hlr_grad(o, m, par, idx):
    par = np.ascontiguousarray(par, np.float64); idx = _idx(idx)
    g = np.zeros(len(idx))
    _hlr_call(o, "hlr_grad", m, None, [_dp, _ip, C.c_int, _dp], dptr(par), iptr(idx), len(idx), dptr(g))
    return g


def hlr_hmc(o, m, par, idx, simlen, eps, seed, it, chain=0, comp=0):
    """One HMC transition; par is updated in place."""
    idx = _idx(idx)
    if o.kind == "ref":
        return _hlr_call(o, "hlr_hmc", m, C.c_int,
                         [_dp, _ip, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32,
                          C.c_uint32], dptr(par), iptr(idx), len(idx), simlen, eps, seed, it, chain, comp)
    L = C.c_int()
    prop = np.zeros(m.D + 2)
    acc = _hlr_call(o, "hlr_hmc", m, C.c_int,
                    [_dp, _ip, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32,
                     C.c_uint32, C.POINTER(C.c_int), _dp],
                    dptr(par), iptr(idx), len(idx), simlen, eps, seed, it, chain, comp, C.byref(L), dptr(prop))
    return acc, L.value, prop


def hlr_rslice(o, m, par, idx, simlen, eps, seed, it, chain=0, comp=0):
    """One reflective-slice transition (cbits/augur_mcmclib.h:498-543); par
    is updated in place.  Returns (moved, simsteps, reflections) for the
    restatement, None for the reference build."""
    idx = _idx(idx)
    if o.kind == "ref":
        _hlr_call(o, "hlr_rslice", m, None,
                  [_dp, _ip, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32],
                  dptr(par), iptr(idx), len(idx), simlen, eps, seed, it, chain, comp)
        return None
    L, R = C.c_int(), C.c_int()
    moved = _hlr_call(o, "hlr_rslice", m, C.c_int,
                      [_dp, _ip, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32,
                       C.c_uint32, C.POINTER(C.c_int), C.POINTER(C.c_int)],
                      dptr(par), iptr(idx), len(idx), simlen, eps, seed, it, chain, comp, C.byref(L), C.byref(R))
    return moved, L.value, R.value


def hlr_nuts(o, m, par, idx, eps, seed, it, chain=0, comp=0, max_depth=64):
    idx = _idx(idx)
    if o.kind == "ref":
        with _quiet_stdout():
            _hlr_call(o, "hlr_nuts", m, None,
                      [_dp, _ip, C.c_int, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32],
                      dptr(par), iptr(idx), len(idx), eps, seed, it, chain, comp)
        return None
    leaves, ovf = C.c_int(), C.c_int()
    depth = _hlr_call(o, "hlr_nuts", m, C.c_int,
                      [_dp, _ip, C.c_int, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                       C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)],
                      dptr(par), iptr(idx), len(idx), eps, seed, it, chain, comp, max_depth,
                      C.byref(leaves), C.byref(ovf))
    return depth, leaves.value, ovf.value


def hlr_mwg(o, m, par, which, var, seed, it, chain=0, comp=0):
    return _hlr_call(o, "hlr_mwg", m, C.c_int,
                     [_dp, C.c_int, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32],
                     dptr(par), which, var, seed, it, chain, comp)


class _quiet_stdout:
    """Silences the C-level stdout (the reference's NUTS prints its stacks)."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        libc = C.CDLL(None)
        libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def hlr_synthetic(N, D, seed, vprior="invgamma", has_b=False, x_dtype=np.float64):
    """Config-style synthetic HLR data: X ~ N(0,1), sigma^2 ~ InvGamma(1,1),
    beta ~ N(0, sigma^2 I), y ~ Bernoulli(sigmoid(X beta (+ b)))."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((N, D)).astype(x_dtype)
    s2 = 1.0 / rng.gamma(1.0, 1.0)
    beta = rng.standard_normal(D) * np.sqrt(s2)
    b = rng.standard_normal() * np.sqrt(s2) if has_b else 0.0
    t = X.astype(np.float64) @ beta + b
    y = (rng.random(N) < 1.0 / (1.0 + np.exp(-t))).astype(np.int32)
    return X, y, beta, s2


# ---- Gaussian mixtures --------------------------------------------------------
class GmmC(C.Structure):
    _fields_ = [("N", C.c_int), ("d", C.c_int), ("K", C.c_int), ("shared_cov", C.c_int),
                ("Y", _dp), ("mu0", _dp), ("cov0", _dp), ("alpha", _dp), ("df", C.c_int),
                ("scale0", _dp)]


class GmmModel:
    """mvgmm (shared covariance `covs`, fixed weights) when shared_cov, else
    hmvgmm (weights ~ Dir(alpha), covariances ~ InvWishart(df, scale0))."""

    def __init__(self, Y, K, mu0, cov0, shared_cov, alpha=None, df=0, scale0=None):
        self.Y = np.ascontiguousarray(Y, np.float64)
        self.N, self.d = self.Y.shape
        self.K = int(K)
        self.mu0 = np.ascontiguousarray(mu0, np.float64)
        self.cov0 = np.ascontiguousarray(cov0, np.float64)
        self.shared = int(bool(shared_cov))
        self.alpha = np.ascontiguousarray(alpha if alpha is not None else np.ones(K), np.float64)
        self.df = int(df)
        self.scale0 = np.ascontiguousarray(scale0 if scale0 is not None else np.eye(self.d), np.float64)

    def struct(self):
        return GmmC(self.N, self.d, self.K, self.shared, dptr(self.Y), dptr(self.mu0), dptr(self.cov0),
                    dptr(self.alpha), self.df, dptr(self.scale0))


def _gmm(o, name, g, restype, types, *args):
    f = o.fn(name, restype)
    f.argtypes = [C.POINTER(GmmC)] + types
    s = g.struct()
    return f(C.byref(s), *args)


_S = [C.c_uint64, C.c_uint32]


def gmm_disc_z(o, g, pis, mu, cov, seed, it):
    z = np.zeros(g.N, np.int32)
    _gmm(o, "gmm_disc_z", g, None, [_dp, _dp, _dp, _ip] + _S, dptr(np.ascontiguousarray(pis, np.float64)),
         dptr(np.ascontiguousarray(mu, np.float64)), dptr(np.ascontiguousarray(cov, np.float64)), iptr(z),
         seed, it)
    return z


def gmm_disc_z_subset(o, g, pis, mu, cov, idx, seed, it):
    """Assignments of the points idx only, each from its own substream (the
    values gmm_disc_z gives those points)."""
    idx = np.ascontiguousarray(idx, np.int32)
    z = np.zeros(len(idx), np.int32)
    _gmm(o, "gmm_disc_z_subset", g, None, [_dp, _dp, _dp, _ip, C.c_int, _ip] + _S,
         dptr(np.ascontiguousarray(pis, np.float64)), dptr(np.ascontiguousarray(mu, np.float64)),
         dptr(np.ascontiguousarray(cov, np.float64)), iptr(idx), len(idx), iptr(z), seed, it)
    return z


def gmm_stats(o, g, z, mu):
    cnt = np.zeros(g.K, np.int32)
    s = np.zeros((g.K, g.d))
    obs = np.zeros((g.K, g.d, g.d))
    _gmm(o, "gmm_stats", g, None, [_ip, _dp, _ip, _dp, _dp], iptr(np.ascontiguousarray(z, np.int32)),
         dptr(np.ascontiguousarray(mu, np.float64)), iptr(cnt), dptr(s), dptr(obs))
    return cnt, s, obs


def gmm_sweep(o, g, pis, mu, cov, z, seed, it):
    """One sweep in place (arrays must be float64 / int32 contiguous)."""
    _gmm(o, "gmm_sweep", g, None, [_dp, _dp, _dp, _ip] + _S, dptr(pis), dptr(mu), dptr(cov), iptr(z), seed, it)


def gmm_conj_pis(o, g, cnt, seed, it):
    pis = np.zeros(g.K)
    _gmm(o, "gmm_conj_pis", g, None, [_ip, _dp] + _S, iptr(np.ascontiguousarray(cnt, np.int32)), dptr(pis), seed, it)
    return pis


def gmm_conj_mu(o, g, cnt, s, cov, seed, it):
    mu = np.zeros((g.K, g.d))
    s = np.array(s, np.float64, copy=True)
    _gmm(o, "gmm_conj_mu", g, None, [_ip, _dp, _dp, _dp] + _S, iptr(np.ascontiguousarray(cnt, np.int32)),
         dptr(s), dptr(np.ascontiguousarray(cov, np.float64)), dptr(mu), seed, it)
    return mu


def gmm_conj_cov(o, g, cnt, obs, seed, it):
    cov = np.zeros((g.K, g.d, g.d))
    obs = np.array(obs, np.float64, copy=True)
    _gmm(o, "gmm_conj_cov", g, None, [_ip, _dp, _dp] + _S, iptr(np.ascontiguousarray(cnt, np.int32)),
         dptr(obs), dptr(cov), seed, it)
    return cov


def gmm_eslice(o, g, mu, cov, z, seed, it):
    mu = np.array(mu, np.float64, copy=True)
    _gmm(o, "gmm_eslice", g, C.c_int if o.kind == "oracle" else None, [_dp, _dp, _ip] + _S, dptr(mu),
         dptr(np.ascontiguousarray(cov, np.float64)), iptr(np.ascontiguousarray(z, np.int32)), seed, it)
    return mu


def gmm_mwg(o, g, mu, cov, z, covp, seed, it, compat=True):
    mu = np.array(mu, np.float64, copy=True)
    covp = np.ascontiguousarray(covp, np.float64)
    zc = np.ascontiguousarray(z, np.int32)
    cv = np.ascontiguousarray(cov, np.float64)
    if o.kind == "ref":
        _gmm(o, "gmm_mwg", g, None, [_dp, _dp, _ip, _dp] + _S, dptr(mu), dptr(cv), iptr(zc), dptr(covp), seed, it)
    else:
        _gmm(o, "gmm_mwg", g, C.c_int, [_dp, _dp, _ip, _dp, C.c_int] + _S, dptr(mu), dptr(cv), iptr(zc),
             dptr(covp), int(compat), seed, it)
    return mu


def gmm_ll_mu(o, g, muk, k, cov, z):
    return _gmm(o, "gmm_ll_mu", g, C.c_double, [_dp, C.c_int, _dp, _ip],
                dptr(np.ascontiguousarray(muk, np.float64)), k, dptr(np.ascontiguousarray(cov, np.float64)),
                iptr(np.ascontiguousarray(z, np.int32)))


def gmm_ll_mod(o, g, pis, mu, cov, z):
    """The model log density augur_get_curr_ll returns for hmvgmm.rv / mvgmm.rv."""
    c = np.ascontiguousarray
    return _gmm(o, "gmm_ll_mod", g, C.c_double, [_dp, _dp, _dp, _ip], dptr(c(pis, np.float64)),
                dptr(c(mu, np.float64)), dptr(c(cov, np.float64)), iptr(c(z, np.int32)))


def gmm_pred_ll(o, Y, pis, mu, cov, shared_cov=False):
    """Test-point log-likelihood of one (pis, mu, cov) sample (oracle only)."""
    c = np.ascontiguousarray
    Y = c(Y, np.float64)
    f = o.fn("gmm_pred_ll", C.c_double)
    f.argtypes = [C.c_int] * 4 + [_dp, _dp, _dp, _dp]
    return f(Y.shape[0], Y.shape[1], len(pis), int(shared_cov), dptr(Y), dptr(c(pis, np.float64)),
             dptr(c(mu, np.float64)), dptr(c(cov, np.float64)))


def mvnormal_ll(o, pt, mean, cov):
    f = o.fn("mvnormal_ll", C.c_double)
    f.argtypes = [_dp, _dp, _dp, C.c_int]
    return f(dptr(np.ascontiguousarray(pt, np.float64)), dptr(np.ascontiguousarray(mean, np.float64)),
             dptr(np.ascontiguousarray(cov, np.float64)), len(pt))


def gmm_synthetic(N, K, d, seed, mean_scale=5.0, df_extra=2, y_dtype=np.float32):
    """Config-style mixture data: means ~ N(0, mean_scale^2 I), covariances ~
    Wishart(d + df_extra, I), weights ~ Dirichlet(1); y stored as float32
    (values exactly representable in binary64)."""
    rng = np.random.default_rng(seed)
    mus = rng.standard_normal((K, d)) * mean_scale
    covs = []
    for _ in range(K):
        A = rng.standard_normal((d + df_extra, d))
        covs.append(A.T @ A / (d + df_extra))
    pis = rng.dirichlet(np.ones(K))
    z = rng.choice(K, size=N, p=pis)
    Y = np.empty((N, d))
    for k in range(K):
        m = z == k
        if m.any():
            Lc = np.linalg.cholesky(covs[k])
            Y[m] = mus[k] + rng.standard_normal((m.sum(), d)) @ Lc.T
    return Y.astype(y_dtype).astype(np.float64), z.astype(np.int32), mus, np.array(covs), pis
