"""The model-handle C ABI driven through ctypes alone, the way a C caller or
the reference's own ctypes front end would bind it: numpy host buffers in
and out, every device buffer allocated by the library, no torch on that
side.  The handles reproduce what the AugurInfer front end samples for the
same model, data, initial point and seed, bit for bit; checkpoint / restore
continues a chain exactly; per-handle errors are reported."""
import ctypes as C
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "augurv2_b200", "_lib", "libaugur_b200.so")
GOLD = os.path.join(HERE, "golden")

i32, u32, u64, f64, sz, vp = C.c_int, C.c_uint32, C.c_uint64, C.c_double, C.c_size_t, C.c_void_p
dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


class LdaInit(C.Structure):
    _fields_ = [("D", i32), ("K", i32), ("V", i32), ("doc_off", ip), ("w", ip), ("alpha", dp), ("beta", dp),
                ("theta", dp), ("phi", dp), ("z", ip), ("seed", u64), ("iter0", u32)]


class HlrComp(C.Structure):
    _fields_ = [("kind", i32), ("P", i32), ("idx_off", i32), ("max_depth", i32), ("simlen", f64), ("eps", f64),
                ("mwg_var", f64)]


class HlrInit(C.Structure):
    _fields_ = [("N", i32), ("D", i32), ("has_b", i32), ("vprior", i32), ("compat", i32), ("lam", f64),
                ("a0", f64), ("s0", f64), ("X", dp), ("y", ip), ("C", i32), ("pars", dp), ("n_comps", i32),
                ("comps", C.POINTER(HlrComp)), ("idx", ip), ("n_idx", i32), ("seed", u64), ("iter0", u32)]


class GmmInit(C.Structure):
    _fields_ = [("N", i32), ("d", i32), ("K", i32), ("shared_cov", i32), ("move", i32), ("compat", i32),
                ("Y", dp), ("mu0", dp), ("cov0", dp), ("pis", dp), ("covs", dp), ("alpha", dp), ("df", i32),
                ("scale0", dp), ("prop_cov", dp), ("mu", dp), ("z", ip), ("seed", u64), ("iter0", u32)]


@pytest.fixture(scope="module")
def L():
    lib = C.CDLL(LIB_PATH)
    sig = {
        "ab_init_lda": (i32, [C.POINTER(LdaInit), C.POINTER(vp)]),
        "ab_init_hlr": (i32, [C.POINTER(HlrInit), C.POINTER(vp)]),
        "ab_init_gmm": (i32, [C.POINTER(GmmInit), C.POINTER(vp)]),
        "ab_step": (i32, [vp, i32, vp]),
        "ab_iteration": (u32, [vp]),
        "ab_state_bytes": (sz, [vp]),
        "ab_get_state": (i32, [vp, vp, sz, vp]),
        "ab_set_state": (i32, [vp, vp, sz, vp]),
        "ab_checkpoint_bytes": (sz, [vp]),
        "ab_checkpoint": (i32, [vp, vp, sz, vp]),
        "ab_restore": (i32, [vp, vp, sz, vp]),
        "ab_curr_ll_count": (i32, [vp]),
        "ab_curr_ll": (i32, [vp, dp, i32, vp]),
        "ab_model_kind": (i32, [vp]),
        "ab_model_last_error": (C.c_char_p, [vp]),
        "ab_destroy": (i32, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


def P(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def ok(L, h, rc):
    assert rc == 0, L.ab_model_last_error(h)


def get_state(L, h):
    buf = np.zeros(L.ab_state_bytes(h), np.uint8)
    ok(L, h, L.ab_get_state(h, buf.ctypes.data, buf.nbytes, None))
    return buf


def lda_split(buf, D, K, V):
    theta = buf[:8 * D * K].view(np.float64).reshape(D, K)
    phi = buf[8 * D * K:8 * (D * K + K * V)].view(np.float64).reshape(K, V)
    z = buf[8 * (D * K + K * V):].view(np.int32)
    return theta, phi, z


def lda_handle(L, off, w, alpha, beta, seed, K, V):
    off, w = np.ascontiguousarray(off, np.int32), np.ascontiguousarray(w, np.int32)
    alpha, beta = np.ascontiguousarray(alpha, np.float64), np.ascontiguousarray(beta, np.float64)
    init = LdaInit(len(off) - 1, K, V, P(off, C.c_int), P(w, C.c_int), P(alpha, C.c_double), P(beta, C.c_double),
                   None, None, None, seed, 0)
    h = vp()
    assert L.ab_init_lda(C.byref(init), C.byref(h)) == 0
    assert L.ab_model_kind(h) == 1
    return h


def test_lda_handle_reproduces_augurinfer_and_the_reference(L):
    """examples/lda.py's corpus (d4_k4_v8) with the default initial point and
    seed 0: ten handle steps give the reference's own assignments and
    proportions (golden fixture) and AugurInfer's samples bit for bit."""
    from augurv2_b200.augurdistlib import AugurDefault
    from augurv2_b200.augurlib import AugurInfer, AugurOpt
    g = np.load(os.path.join(GOLD, "lda_d4_k4_v8.npz"))
    off, w = g["doc_off"], g["w"]
    D, K, V = 4, 4, 8
    h = lda_handle(L, off, w, g["alpha"], g["beta"], 0, K, V)
    got = []
    for it in range(10):
        ok(L, h, L.ab_step(h, 1, None))
        got.append([a.copy() for a in lda_split(get_state(L, h), D, K, V)])
        np.testing.assert_array_equal(got[-1][2], g["z"][it])
        np.testing.assert_allclose(got[-1][0], g["theta"][it], rtol=1e-12)
    assert L.ab_iteration(h) == 10
    ll = np.zeros(1)
    ok(L, h, L.ab_curr_ll(h, P(ll, C.c_double), 1, None))
    assert np.isfinite(ll[0])
    L.ab_destroy(h)
    models = json.load(open(os.path.join(GOLD, "models.json")))
    rec = models["examples"]["lda"]
    with AugurInfer("config.yml", rec["model"]) as infer:
        infer.set_compile_opt(AugurOpt(cached=False, target="cpu", initStrat=AugurDefault()))
        infer.set_user_sched(rec["scheds"][0])
        infer.compile(K, D, np.diff(off).astype(np.int32), g["alpha"], g["beta"])(
            [w[off[d]:off[d + 1]] for d in range(D)])
        s = infer.samplen(burnIn=0, numSamples=10)
        front_ll = infer.curr_ll()
    for it in range(10):
        np.testing.assert_array_equal(np.concatenate(s["z"][it]), got[it][2])
        np.testing.assert_array_equal(s["theta"][it], got[it][0])
        np.testing.assert_array_equal(s["phi"][it], got[it][1])
    assert front_ll == ll[0]


def test_hlr_handle_reproduces_augurinfer(L):
    from augurv2_b200.augurlib import AugurInfer, AugurOpt
    from oracle import oracle as O
    models = json.load(open(os.path.join(GOLD, "models.json")))
    rec = models["examples"]["hlr"]
    N, D = 500, 6
    X, y, beta, s2 = O.hlr_synthetic(N, D, 3, has_b=True)
    sched = rec["scheds"][1]        # MWG [v] (*) MWG [b] (*) HMC [theta] [0.5, 0.05]
    with AugurInfer("config.yml", rec["model"]) as infer:
        infer.set_compile_opt(AugurOpt(cached=False, target="cpu", seed=1))
        infer.set_user_sched(sched)
        infer.compile(D, N, 1.0, X)(y)
        init = infer.backend.chains.state().copy()
        s = infer.samplen(burnIn=0, numSamples=12)
        front_ll = infer.curr_ll()
    X = np.ascontiguousarray(X, np.float64)
    y = np.ascontiguousarray(y, np.int32)
    idx = np.array([D + 1, D] + list(range(D)), np.int32)
    comps = (HlrComp * 3)(HlrComp(2, 1, 0, 0, 0.0, 0.0, 1.0), HlrComp(2, 1, 1, 0, 0.0, 0.0, 1.0),
                          HlrComp(0, D, 2, 0, 0.5, 0.05, 0.0))
    pars = np.ascontiguousarray(init, np.float64)
    hi = HlrInit(N, D, 1, 0, 1, 1.0, 1.0, 1.0, P(X, C.c_double), P(y, C.c_int), 1, P(pars, C.c_double), 3,
                 comps, P(idx, C.c_int), len(idx), 1, 0)
    h = vp()
    assert L.ab_init_hlr(C.byref(hi), C.byref(h)) == 0
    for it in range(12):
        ok(L, h, L.ab_step(h, 1, None))
        st = get_state(L, h).view(np.float64).reshape(1, D + 2)
        np.testing.assert_array_equal(st[0, :D], s["theta"][it])
        assert st[0, D] == s["b"][it] and st[0, D + 1] == s["v"][it]
    ll = np.zeros(1)
    assert L.ab_curr_ll_count(h) == 1
    ok(L, h, L.ab_curr_ll(h, P(ll, C.c_double), 1, None))
    assert ll[0] == front_ll
    L.ab_destroy(h)


def test_checkpoint_restore_continues_exactly(L):
    from augurv2_b200.lda import synthetic_corpus
    K, V = 10, 120
    off, w = synthetic_corpus(K, V, 30, 25, 0.2, 0.05, seed=4)
    a = lda_handle(L, off, w, np.full(K, 0.2), np.full(V, 0.05), 11, K, V)
    ok(L, a, L.ab_step(a, 3, None))
    ck = np.zeros(L.ab_checkpoint_bytes(a), np.uint8)
    ok(L, a, L.ab_checkpoint(a, ck.ctypes.data, ck.nbytes, None))
    ok(L, a, L.ab_step(a, 4, None))
    want = get_state(L, a)
    b = lda_handle(L, off, w, np.full(K, 0.2), np.full(V, 0.05), 11, K, V)
    ok(L, b, L.ab_restore(b, ck.ctypes.data, ck.nbytes, None))
    assert L.ab_iteration(b) == 3
    ok(L, b, L.ab_step(b, 4, None))
    np.testing.assert_array_equal(get_state(L, b), want)
    # a checkpoint of another model is refused, with the message on the handle
    c = lda_handle(L, off, w, np.full(K, 0.2), np.full(V, 0.05), 12, K, V)
    assert L.ab_restore(c, ck.ctypes.data, ck.nbytes, None) == 1
    assert b"seed" in L.ab_model_last_error(c)
    assert L.ab_get_state(c, ck.ctypes.data, 3, None) == 1
    assert b"bytes" in L.ab_model_last_error(c)
    for h in (a, b, c):
        L.ab_destroy(h)


def test_gmm_handle_matches_gmmgibbs_and_restores(L):
    from augurv2_b200.gmm import GmmGibbs
    from oracle import oracle as O
    N_, K, d = 1500, 4, 5
    Y, z, mus, covs, pis = O.gmm_synthetic(N_, K, d, seed=11)
    Y = np.ascontiguousarray(Y, np.float64)
    mu0, cov0, alpha, scale0 = np.zeros(d), 25 * np.eye(d), np.ones(K), np.eye(d)
    ref = GmmGibbs(Y, K, mu0, cov0, alpha=alpha, df=d + 2, scale0=scale0, mu=mus, cov=covs, pis=pis, z=z, seed=3)
    arrs = [np.ascontiguousarray(a, np.float64) for a in (mu0, cov0, pis, covs, alpha, scale0, mus)]
    zc = np.ascontiguousarray(z, np.int32)
    gi = GmmInit(N_, d, K, 0, 0, 1, P(Y, C.c_double), *[P(a, C.c_double) for a in arrs[:5]], d + 2,
                 P(arrs[5], C.c_double), None, P(arrs[6], C.c_double), P(zc, C.c_int), 3, 0)
    h = vp()
    assert L.ab_init_gmm(C.byref(gi), C.byref(h)) == 0
    for it in range(3):
        ref.sweep(1)
        ok(L, h, L.ab_step(h, 1, None))
        buf = get_state(L, h)
        o = 0
        st = ref.state()
        for name, n in (("pis", K), ("mu", K * d), ("cov", K * d * d)):
            np.testing.assert_array_equal(buf[o:o + 8 * n].view(np.float64), st[name].ravel())
            o += 8 * n
        np.testing.assert_array_equal(buf[o:].view(np.int32), st["z"])
    ll = np.zeros(1)
    ok(L, h, L.ab_curr_ll(h, P(ll, C.c_double), 1, None))
    assert ll[0] == ref.ll_mod()
    ck = np.zeros(L.ab_checkpoint_bytes(h), np.uint8)
    ok(L, h, L.ab_checkpoint(h, ck.ctypes.data, ck.nbytes, None))
    ok(L, h, L.ab_step(h, 2, None))
    want = get_state(L, h)
    ok(L, h, L.ab_restore(h, ck.ctypes.data, ck.nbytes, None))
    ok(L, h, L.ab_step(h, 2, None))
    np.testing.assert_array_equal(get_state(L, h), want)
    L.ab_destroy(h)
