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
