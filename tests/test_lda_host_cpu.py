"""Host logic of the LDA sampler that needs no GPU: the packed sample layout
behind LdaGibbs.samples (one transfer per sample) and the corpus
flattening."""
import types

import numpy as np
import torch

from augurv2_b200.lda import LdaGibbs, flatten_docs


def _fake(D, K, V, T):
    o = types.SimpleNamespace(D=D, K=K, V=V, T=T)
    o._sample_layout = lambda: LdaGibbs._sample_layout(o)
    return o


def test_packed_sample_layout_is_aligned_and_disjoint():
    for D, K, V, T in [(3, 5, 7, 11), (2000, 50, 10000, 399614), (1, 1, 1, 0)]:
        o = _fake(D, K, V, T)
        (ot, op, oz), nbytes = LdaGibbs._sample_layout(o)
        assert ot == 0 and op % 256 == 0 and oz % 256 == 0 and nbytes % 256 == 0
        assert op >= 8 * D * K and oz >= op + 8 * K * V and nbytes >= oz + 4 * T
        buf = torch.zeros(nbytes, dtype=torch.uint8)
        th, ph, z = LdaGibbs._sample_views(o, buf)
        assert th.shape == (D, K) and ph.shape == (K, V) and z.shape == (T,)
        assert th.dtype == torch.float64 and ph.dtype == torch.float64 and z.dtype == torch.int32
        th.fill_(1.5)
        ph.fill_(-2.0)
        z.fill_(7)
        th2, ph2, z2 = LdaGibbs._sample_views(o, buf)
        assert float(th2.sum()) == 1.5 * D * K and float(ph2.sum()) == -2.0 * K * V and int(z2.sum()) == 7 * T


def test_flatten_docs_csr():
    off, w = flatten_docs([[1, 2, 3], [], [4], np.array([5, 6])])
    assert off.tolist() == [0, 3, 3, 4, 6] and w.tolist() == [1, 2, 3, 4, 5, 6]
    assert off.dtype == np.int32 and w.dtype == np.int32
