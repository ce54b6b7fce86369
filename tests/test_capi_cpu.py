"""The C-ABI library loads without a GPU, exports every symbol that
include/augur_b200.h declares, and rejects bad arguments with a status and a
message (no compute calls are made here)."""
import ctypes as C

import pytest

from augurv2_b200 import _native as N


def test_library_exports_header_symbols():
    L = N.lib()
    syms = N.header_symbols()
    assert len(syms) > 5
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_every_header_symbol_has_a_ctypes_signature():
    missing = [s for s in N.header_symbols() if s not in N._SIGS]
    assert not missing, missing


def test_version_and_error_string():
    assert b"sm_100a" in N.lib().ab_version()
    assert isinstance(N.last_error(), str)


@pytest.mark.parametrize("D,K,V", [(0, 4, 8), (4, 0, 8), (4, 4, 0), (4, 5000, 8)])
def test_lda_bad_sizes_rejected(D, K, V):
    rc = N.lib().ab_lda_count(D, K, V, None, None, None, None, None, None)
    assert rc == 1
    assert "LDA" in N.last_error()


def test_lda_null_pointer_rejected():
    rc = N.lib().ab_lda_disc_z(4, 4, 8, None, None, None, None, None, None, None, 0, 0, None)
    assert rc == 1 and "null" in N.last_error()


def test_lda_create_requires_every_pointer():
    d = N.LdaDesc(4, 4, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    h = C.c_void_p()
    assert N.lib().ab_lda_create(C.byref(d), C.byref(h)) == 1


def test_model_handle_arguments_checked_before_any_device_work():
    """ab_init_* validates the host descriptor before it allocates: a token
    id outside [0, V), a block index outside the parameters or a bad move
    are refused with a status and a message."""
    import numpy as np
    L = N.lib()
    off = np.array([0, 2, 3], np.int32)
    w = np.array([0, 7, 1], np.int32)            # 7 >= V = 5
    a, b = np.ones(2), np.ones(5)
    P = lambda x, t: x.ctypes.data_as(C.POINTER(t))
    d = N.LdaInit(2, 2, 5, P(off, C.c_int), P(w, C.c_int), P(a, C.c_double), P(b, C.c_double), None, None, None,
                  0, 0)
    h = C.c_void_p()
    assert L.ab_init_lda(C.byref(d), C.byref(h)) == 1 and "outside [0, V)" in N.last_error()
    X, y, pars = np.zeros((3, 2)), np.zeros(3, np.int32), np.zeros((1, 4))
    idx = np.array([0, 9], np.int32)                 # 9 >= D + 2
    comps = (N.HlrCompC * 1)(N.HlrCompC(0, 2, 0, 0, 0.5, 0.05, 0.0))
    hi = N.HlrInit(3, 2, 1, 0, 1, 1.0, 1.0, 1.0, P(X, C.c_double), P(y, C.c_int), 1, P(pars, C.c_double), 1,
                   comps, P(idx, C.c_int), 2, 0, 0)
    assert L.ab_init_hlr(C.byref(hi), C.byref(h)) == 1 and "block index" in N.last_error()
    Y, z = np.zeros((3, 2)), np.zeros(3, np.int32)
    m = np.zeros(2)
    c2 = np.eye(2)
    gi = N.GmmInit(3, 2, 1, 1, 1, 1, P(Y, C.c_double), P(m, C.c_double), P(c2, C.c_double), P(np.ones(1), C.c_double),
                   P(c2, C.c_double), None, 0, None, None, P(m, C.c_double), P(z, C.c_int), 0, 0)
    gi.move = 2                                      # MWG without a proposal covariance
    assert L.ab_init_gmm(C.byref(gi), C.byref(h)) == 1 and "prop_cov" in N.last_error()
    assert L.ab_step(None, 1, None) == 1
    assert L.ab_state_bytes(None) == 0 and L.ab_model_last_error(None) == b""
