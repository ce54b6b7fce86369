"""GPU parity of the LDA Gibbs path against the CPU oracle.

Contract (per sweep): given the same theta, phi and Philox uniforms, the
assignments z and both count tables equal the reference CPU sampler's bit for
bit; theta and phi (gamma draws through CUDA's log/pow, phi normalised by a
tree sum) agree to 1e-12 relative.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from augurv2_b200 import _native as N
from augurv2_b200.lda import LdaGibbs, synthetic_corpus
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
RTOL = 1e-12


@pytest.fixture(scope="module")
def orc():
    return O.Oracle("oracle")


def dev(a, dt):
    return torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dt)


def random_problem(seed, D=150, K=50, V=700, mean_len=80):
    rng = np.random.default_rng(seed)
    lens = rng.poisson(mean_len, size=D)
    lens[::17] = 0                                   # empty documents
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    w = rng.integers(0, V, size=off[-1]).astype(np.int32)
    theta = rng.dirichlet(np.full(K, 0.3), size=D)
    phi = rng.dirichlet(np.full(V, 0.05), size=K)
    return off, w, theta, phi


def phiT_of(phi):
    K, V = phi.shape
    Kp = N.lib().ab_lda_phi_stride(K)
    out = np.zeros((V, Kp))
    out[:, :K] = phi.T
    return out, Kp


@pytest.mark.parametrize("seed,K,V", [(0, 50, 700), (1, 50, 700), (2, 1, 30), (3, 2, 30), (4, 3, 40),
                                      (5, 17, 90), (6, 64, 300), (7, 200, 500), (8, 1024, 64),
                                      (9, 65, 200), (10, 100, 300), (11, 128, 90), (12, 256, 400),
                                      (13, 257, 100), (14, 8, 20), (15, 9, 50)])
def test_disc_z_and_counts_bit_exact(orc, seed, K, V):
    off, w, theta, phi = random_problem(seed, D=60 if K > 100 else 150, K=K, V=V)
    if seed % 3 == 2:                                 # exact zeros in theta and phi
        theta[:, ::3] = 0.0
        theta[theta.sum(1) == 0, 0] = 1.0
        phi[::2, ::5] = 0.0
    D, K = theta.shape
    V = phi.shape[1]
    phiT, _ = phiT_of(phi)
    z = torch.zeros(len(w), dtype=torch.int32, device="cuda")
    cdk = torch.zeros((D, K), dtype=torch.int32, device="cuda")
    ckw = torch.zeros((K, V), dtype=torch.int32, device="cuda")
    g = [dev(off, torch.int32), dev(w, torch.int32), dev(theta, torch.float64), dev(phiT, torch.float64)]
    N.check(N.lib().ab_lda_disc_z(D, K, V, N.ptr(g[0]), N.ptr(g[1]), N.ptr(g[2]), N.ptr(g[3]),
                                  N.ptr(z), N.ptr(cdk), N.ptr(ckw), 42, 9, N.stream_ptr()), "disc_z")
    z_ref = orc.lda_disc_z(off, w, theta, phi, np.zeros(len(w), np.int32), 42, 9)
    np.testing.assert_array_equal(z.cpu().numpy(), z_ref)
    c_dk, c_kw = orc.lda_conj_stat(off, w, z_ref, D, K, V)
    np.testing.assert_array_equal(cdk.cpu().numpy(), c_dk)
    np.testing.assert_array_equal(ckw.cpu().numpy(), c_kw)


@pytest.mark.parametrize("K", [50, 100, 200, 300])
def test_disc_z_degenerate_norms(orc, K):
    """Tokens whose normaliser is zero, subnormal or tiny (the division-free
    test cannot decide them) take the reference's own loop: still bit-exact."""
    off, w, theta, phi = random_problem(20 + K, D=40, K=K, V=120)
    theta[1::4] *= 1e-300            # products underflow to subnormals or zero
    theta[2::4] *= 1e-150            # norm near 1e-150 * phi: tiny but normal
    phi[:, 7] = 0.0                  # word 7: every product zero, norm 0
    phi[:, 9] = 1e-310               # word 9: subnormal phi entries
    D, K = theta.shape
    V = phi.shape[1]
    phiT, _ = phiT_of(phi)
    z = torch.zeros(len(w), dtype=torch.int32, device="cuda")
    g = [dev(off, torch.int32), dev(w, torch.int32), dev(theta, torch.float64), dev(phiT, torch.float64)]
    N.check(N.lib().ab_lda_disc_z(D, K, V, N.ptr(g[0]), N.ptr(g[1]), N.ptr(g[2]), N.ptr(g[3]),
                                  N.ptr(z), None, None, 3, 1, N.stream_ptr()), "disc_z")
    z_ref = orc.lda_disc_z(off, w, theta, phi, np.zeros(len(w), np.int32), 3, 1)
    np.testing.assert_array_equal(z.cpu().numpy(), z_ref)


def test_count_kernel(orc):
    off, w, theta, phi = random_problem(3)
    D, K = theta.shape
    V = phi.shape[1]
    z = np.random.default_rng(3).integers(0, K, size=len(w)).astype(np.int32)
    cdk = torch.full((D, K), 7, dtype=torch.int32, device="cuda")
    ckw = torch.full((K, V), 7, dtype=torch.int32, device="cuda")
    g = [dev(off, torch.int32), dev(w, torch.int32), dev(z, torch.int32)]  # keep alive
    N.check(N.lib().ab_lda_count(D, K, V, N.ptr(g[0]), N.ptr(g[1]), N.ptr(g[2]), N.ptr(cdk), N.ptr(ckw),
                                 N.stream_ptr()), "count")
    c_dk, c_kw = orc.lda_conj_stat(off, w, z, D, K, V)
    np.testing.assert_array_equal(cdk.cpu().numpy(), c_dk)
    np.testing.assert_array_equal(ckw.cpu().numpy(), c_kw)


def test_conj_theta_matches_oracle(orc):
    rng = np.random.default_rng(5)
    D, K = 300, 50
    cnt = rng.poisson(3.0, size=(D, K)).astype(np.int32)
    cnt[::7] = 0
    alpha = np.full(K, 0.1)
    out = torch.zeros((D, K), dtype=torch.float64, device="cuda")
    g = [dev(alpha, torch.float64), dev(cnt, torch.int32)]  # keep alive
    N.check(N.lib().ab_lda_conj_theta(D, K, N.ptr(g[0]), N.ptr(g[1]), N.ptr(out), 77, 4, N.stream_ptr()),
            "conj_theta")
    ref = orc.lda_conj_theta(alpha, cnt, 77, 4)
    got = out.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=RTOL, atol=0)
    np.testing.assert_allclose(got.sum(1), 1.0, rtol=1e-12)


@pytest.mark.parametrize("K,V", [(50, 1000), (3, 37), (7, 4)])
def test_conj_phi_matches_oracle(orc, K, V):
    rng = np.random.default_rng(K * V)
    cnt = rng.poisson(1.0, size=(K, V)).astype(np.int32)
    beta = np.full(V, 0.01)
    phiT, Kp = phiT_of(np.zeros((K, V)))
    ckw = dev(cnt, torch.int32)
    out = dev(phiT, torch.float64)
    bt = dev(beta, torch.float64)  # keep alive
    scratch = torch.full((int(N.lib().ab_lda_phi_scratch_bytes(K, V)),), 0xAB, dtype=torch.uint8,
                         device="cuda")
    N.check(N.lib().ab_lda_conj_phi(K, V, N.ptr(bt), N.ptr(ckw), N.ptr(out), 1, 55, 2, N.ptr(scratch),
                                    N.stream_ptr()), "conj_phi")
    ref = orc.lda_conj_phi(beta, cnt, 55, 2)
    got = out.cpu().numpy()[:, :K].T
    np.testing.assert_allclose(got, ref, rtol=RTOL, atol=1e-300)
    assert (ckw.cpu().numpy() == 0).all(), "clear_counts must zero the table"


def per_sweep_contract(orc, s, off, w, alpha, beta, z_prev, theta, phi, z, seed, it):
    D, K = theta.shape
    V = phi.shape[1]
    c_dk, c_kw = orc.lda_conj_stat(off, w, z_prev, D, K, V)
    np.testing.assert_allclose(theta, orc.lda_conj_theta(alpha, c_dk, seed, it), rtol=RTOL, atol=0)
    np.testing.assert_allclose(phi, orc.lda_conj_phi(beta, c_kw, seed, it), rtol=RTOL, atol=1e-300)
    z_ref = orc.lda_disc_z(off, w, theta, phi, np.zeros_like(z), seed, it)
    np.testing.assert_array_equal(z, z_ref, err_msg="sweep %d" % s)


def test_sweep_runner_reference_fixture(orc):
    """The reference's own example corpus (examples/lda.py d4_k4_v8): the
    graph-replayed sweeps meet the per-sweep contract and reproduce the
    reference's assignments for all 10 sweeps."""
    g = np.load(os.path.join(GOLD, "lda_d4_k4_v8.npz"))
    K, V = 4, 8
    s = LdaGibbs(K, V, g["doc_off"], g["w"], g["alpha"], g["beta"], seed=0)
    z_prev = np.zeros(len(g["w"]), np.int32)
    for it in range(10):
        s.sweep(1)
        theta, phi, z = s.state()
        per_sweep_contract(orc, it, g["doc_off"], g["w"], g["alpha"], g["beta"], z_prev, theta, phi, z, 0, it)
        np.testing.assert_array_equal(z, g["z"][it])
        np.testing.assert_allclose(theta, g["theta"][it], rtol=RTOL)
        z_prev = z
    s.close()


@pytest.mark.parametrize("K", [20, 100])
def test_sweep_runner_synthetic_graph_vs_eager(orc, K):
    """K = 20 runs the binary32-screened z kernel and the three-kernel phi
    draw, K = 100 the binary64 kernels; both meet the per-sweep contract."""
    V, D = 500, 60
    off, w = synthetic_corpus(K, V, D, 50, 0.1, 0.01, seed=11)
    alpha, beta = np.full(K, 0.1), np.full(V, 0.01)
    z0 = np.random.default_rng(1).integers(0, K, size=len(w)).astype(np.int32)
    a = LdaGibbs(K, V, off, w, alpha, beta, seed=123, z=z0)
    b = LdaGibbs(K, V, off, w, alpha, beta, seed=123, z=z0)
    z_prev = z0
    for it in range(4):
        a.sweep(1, graph=True)
        b.sweep(1, graph=False)
        sa, sb = a.state(), b.state()
        for x, y in zip(sa, sb):
            np.testing.assert_array_equal(x, y)
        per_sweep_contract(orc, it, off, w, alpha, beta, z_prev, *sa, 123, it)
        z_prev = sa[2]
    # counts held by the runner equal the statistics of the current z
    c_dk, c_kw = orc.lda_conj_stat(off, w, z_prev, D, K, V)
    np.testing.assert_array_equal(a.cnt_dk.cpu().numpy(), c_dk)
    np.testing.assert_array_equal(a.cnt_kw.cpu().numpy(), c_kw)
    a.close(); b.close()


def test_pipelined_samples_equal_sweep_and_state():
    """LdaGibbs.samples (device snapshots copied out on a second stream while
    the next sweeps run) returns what sweep + state() return at the same
    points, and leaves the sampler in the same state."""
    K, V, D = 20, 500, 60
    off, w = synthetic_corpus(K, V, D, 50, 0.1, 0.01, seed=5)
    a = LdaGibbs(K, V, off, w, 0.1, 0.01, seed=9)
    b = LdaGibbs(K, V, off, w, 0.1, 0.01, seed=9)
    got = list(a.samples(6, first=2, every=3))
    assert len(got) == 6
    for i, sa in enumerate(got):
        b.sweep(2 if i == 0 else 3)
        for x, y in zip(sa, b.state()):
            np.testing.assert_array_equal(x, y)
    a.sweep(1)
    b.sweep(1)
    for x, y in zip(a.state(), b.state()):
        np.testing.assert_array_equal(x, y)
    a.close(); b.close()


def test_full_size_properties():
    """Benchmark shape (K=50, V=1e4, D=2000, ~4e5 tokens): every count table
    sums to the token count, rows of theta/phi are distributions, and the
    document counts equal the per-document histogram of z."""
    K, V, D = 50, 10000, 2000
    off, w = synthetic_corpus(K, V, D, 200, 0.1, 0.01, seed=0)
    s = LdaGibbs(K, V, off, w, 0.1, 0.01, seed=0)
    s.sweep(5)
    torch.cuda.synchronize()
    T = len(w)
    assert int(s.cnt_kw.sum()) == T and int(s.cnt_dk.sum()) == T
    theta, phi, z = s.state()
    np.testing.assert_allclose(theta.sum(1), 1.0, rtol=1e-12)
    np.testing.assert_allclose(phi.sum(1), 1.0, rtol=1e-12)
    doc = np.repeat(np.arange(D), np.diff(off))
    hist = np.zeros((D, K), np.int64)
    np.add.at(hist, (doc, z), 1)
    np.testing.assert_array_equal(s.cnt_dk.cpu().numpy(), hist)
    s.close()


def _phi32_of(phi):
    K, V = phi.shape
    Kq = N.lib().ab_lda_phi32_stride(K)
    out = np.zeros((V, Kq), np.float32)
    out[:, :K] = phi.T.astype(np.float32)        # round to nearest binary32
    return out


@pytest.mark.parametrize("seed,K,V,degenerate", [(0, 50, 700, False), (1, 1, 30, False), (2, 2, 30, True),
                                                 (3, 3, 40, False), (4, 4, 50, False), (5, 16, 90, True),
                                                 (6, 32, 300, False), (7, 33, 120, False), (8, 64, 300, True),
                                                 (9, 61, 200, False), (10, 9, 50, False), (11, 50, 700, True)])
def test_disc_z_f32_screen_bit_exact(orc, seed, K, V, degenerate):
    """The binary32-screened z kernel gives the reference's assignments and
    counts bit for bit, including half rows of every length (K = 1..64) and
    tokens the screen cannot decide (exact zeros, products that underflow
    binary32, tiny and zero norms)."""
    off, w, theta, phi = random_problem(seed, D=150, K=K, V=V)
    if degenerate:
        theta[:, ::3] = 0.0
        theta[theta.sum(1) == 0, 0] = 1.0
        theta[1::4] *= 1e-300                 # products below binary32 range, norm 0 in binary32
        theta[2::4] *= 1e-25                  # norm below 2^-60 but normal in binary64
        phi[:, 7 % V] = 0.0
        phi[::2, 1 % V] = 1e-40               # binary32 subnormals
    D = theta.shape[0]
    phiT, _ = phiT_of(phi)
    phi32 = _phi32_of(phi)
    z = torch.zeros(len(w), dtype=torch.int32, device="cuda")
    cdk = torch.zeros((D, K), dtype=torch.int32, device="cuda")
    ckw = torch.zeros((K, V), dtype=torch.int32, device="cuda")
    g = [dev(off, torch.int32), dev(w, torch.int32), dev(theta, torch.float64), dev(phiT, torch.float64),
         torch.as_tensor(phi32).cuda()]
    N.check(N.lib().ab_lda_disc_z_f32(D, K, V, N.ptr(g[0]), N.ptr(g[1]), N.ptr(g[2]), N.ptr(g[3]), N.ptr(g[4]),
                                      N.ptr(z), N.ptr(cdk), N.ptr(ckw), 42, 9, N.stream_ptr()), "disc_z_f32")
    z_ref = orc.lda_disc_z(off, w, theta, phi, np.zeros(len(w), np.int32), 42, 9)
    np.testing.assert_array_equal(z.cpu().numpy(), z_ref)
    c_dk, c_kw = orc.lda_conj_stat(off, w, z_ref, D, K, V)
    np.testing.assert_array_equal(cdk.cpu().numpy(), c_dk)
    np.testing.assert_array_equal(ckw.cpu().numpy(), c_kw)


def test_sweep_phi32_copy_is_phi_rounded():
    """The sweep runner's binary32 copy of phi (the z screen's input) is phi
    rounded to nearest, with zero padding."""
    K, V, D = 50, 600, 40
    off, w = synthetic_corpus(K, V, D, 60, 0.1, 0.01, seed=3)
    s = LdaGibbs(K, V, off, w, 0.1, 0.01, seed=2)
    s.sweep(2)
    torch.cuda.synchronize()
    L = N.lib()
    Kq = L.ab_lda_phi32_stride(K)
    raw = s.scratch.cpu().numpy()
    off32 = (int(L.ab_lda_phi_scratch_bytes(K, V)) + 255) & ~255     # after the phi draw's scratch
    phi32 = raw[off32:off32 + 4 * V * Kq].view(np.float32).reshape(V, Kq)
    phi = s.state()[1]
    np.testing.assert_array_equal(phi32[:, :K], phi.T.astype(np.float32))
    assert (phi32[:, K:] == 0).all()
    s.close()

