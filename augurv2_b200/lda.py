"""LDA Gibbs sampler on the GPU: host side of the ab_lda_* entry points.

Model (compiler/augur/test/lda.rv, examples/lda.py:12-22):
    theta[d] ~ Dirichlet(alpha)            for d < D
    phi[k]   ~ Dirichlet(beta)             for k < K
    z[d, n]  ~ Categorical(theta[d])       for n < N[d]
    w[d, n]  ~ Categorical(phi[z[d, n]])
Schedule: ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z].

Device state lives in torch tensors owned by this object; every sweep runs
as a replay of a captured CUDA graph of four kernels (lda.cu).
"""
import ctypes as C

import numpy as np
import torch

from . import _native as N
from .checkpoint import Checkpointable
from .trace import traced


def flatten_docs(w):
    """Ragged documents (sequence of int arrays, or a 2-D array) -> CSR
    (doc_off int32[D+1], w int32[T]), the flattening of
    cbits/augur_vecop.c:842-941 without per-row headers."""
    docs = [np.asarray(x, dtype=np.int32).ravel() for x in w]
    lens = np.array([len(x) for x in docs], dtype=np.int64)
    off = np.zeros(len(docs) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    if off[-1] >= 2**31:
        raise ValueError("more than 2^31 tokens")
    flat = np.concatenate(docs) if docs else np.zeros(0, np.int32)
    return off.astype(np.int32), flat.astype(np.int32)


class LdaGibbs(Checkpointable):
    # the assignments and the iteration determine the rest (the counts are
    # recounted and theta / phi are redrawn before they are used)
    _ckpt_tensors = ("theta", "phiT", "z", "cnt_dk", "cnt_kw")
    _ckpt_scalars = ("iteration", "seed")

    def _ckpt_after_load(self):
        N.check(N.lib().ab_lda_init_state(self._h, self.iteration, N.stream_ptr()), "ab_lda_init_state")

    def __init__(self, K, V, doc_off, w, alpha, beta, seed=0, theta=None, phi=None, z=None,
                 iter0=0, device="cuda"):
        self.dev = torch.device(device)
        self.K, self.V = int(K), int(V)
        doc_off = np.ascontiguousarray(doc_off, dtype=np.int32)
        w = np.ascontiguousarray(w, dtype=np.int32)
        self.D = len(doc_off) - 1
        self.T = int(doc_off[-1])
        if w.shape[0] != self.T:
            raise ValueError("w has %d tokens, doc_off says %d" % (w.shape[0], self.T))
        if self.T and (w.min() < 0 or w.max() >= self.V):
            raise ValueError("token ids must lie in [0, V)")
        L = N.lib()
        self.Kp = L.ab_lda_phi_stride(self.K)
        self.seed = int(seed)
        t = lambda a, dt: torch.as_tensor(a, dtype=dt).to(self.dev)
        self.doc_off = t(doc_off, torch.int32)
        self.w = t(w, torch.int32)
        self.alpha = t(np.broadcast_to(np.asarray(alpha, np.float64), (self.K,)).copy(), torch.float64)
        self.beta = t(np.broadcast_to(np.asarray(beta, np.float64), (self.V,)).copy(), torch.float64)
        self.theta = torch.empty((self.D, self.K), dtype=torch.float64, device=self.dev)
        self.phiT = torch.zeros((self.V, self.Kp), dtype=torch.float64, device=self.dev)
        self.z = torch.zeros(self.T, dtype=torch.int32, device=self.dev)
        self.cnt_dk = torch.zeros((self.D, self.K), dtype=torch.int32, device=self.dev)
        self.cnt_kw = torch.zeros((self.K, self.V), dtype=torch.int32, device=self.dev)
        self.scratch = torch.zeros(int(L.ab_lda_scratch_bytes(self.K, self.V)), dtype=torch.uint8, device=self.dev)
        # defaults (uniform theta and phi, z = 0) are filled on the device;
        # given values are uploaded
        if theta is None:
            self.theta.fill_(1.0 / self.K)
        if phi is None:
            self.phiT[:, :self.K].fill_(1.0 / self.V)
        self.set_state(theta=theta, phi=phi, z=z, iteration=iter0)
        desc = N.LdaDesc(self.D, self.K, self.V, self.doc_off.data_ptr(), self.w.data_ptr(),
                         self.alpha.data_ptr(), self.beta.data_ptr(), self.z.data_ptr(),
                         self.theta.data_ptr(), self.phiT.data_ptr(), self.cnt_dk.data_ptr(),
                         self.cnt_kw.data_ptr(), self.scratch.data_ptr(), self.seed)
        h = C.c_void_p()
        N.check(L.ab_lda_create(C.byref(desc), C.byref(h)), "ab_lda_create")
        self._h = h
        self._desc = desc
        N.check(L.ab_lda_init_state(self._h, self.iteration, N.stream_ptr()), "ab_lda_init_state")

    # ---- state -------------------------------------------------------------
    def set_state(self, theta=None, phi=None, z=None, iteration=None):
        if theta is not None:
            self.theta.copy_(torch.as_tensor(np.asarray(theta, np.float64).reshape(self.D, self.K)))
        if phi is not None:
            ph = torch.as_tensor(np.asarray(phi, np.float64).reshape(self.K, self.V)).to(self.dev)
            self.phiT[:, :self.K].copy_(ph.t())      # transposed on the device
        if z is not None:
            self.z.copy_(torch.as_tensor(np.asarray(z, np.int32).ravel()))
        if iteration is not None:
            self.iteration = int(iteration)
        if getattr(self, "_h", None) is not None:
            N.check(N.lib().ab_lda_init_state(self._h, self.iteration, N.stream_ptr()),
                    "ab_lda_init_state")

    def state(self, stream=None):
        """(theta [D,K], phi [K,V], z [T]) as host numpy arrays.

        The three copies go asynchronously into page-locked host buffers
        (torch's caching host allocator, so a sample that is dropped gives
        its buffers to the next one) with one synchronisation at the end:
        about 3x less time per sample than three pageable copies."""
        st = stream if stream is not None else torch.cuda.current_stream(self.dev)
        with torch.cuda.stream(st):
            phi = self.phiT[:, :self.K].t().contiguous()
            out = []
            for t in (self.theta, phi, self.z):
                h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                h.copy_(t, non_blocking=True)
                out.append(h)
        st.synchronize()
        return tuple(h.numpy() for h in out)

    def _sample_layout(self):
        """Byte offsets of theta, phi [K][V] and z in one packed sample."""
        def al(x):
            return (x + 255) & ~255
        nt, nphi, nz = 8 * self.D * self.K, 8 * self.K * self.V, 4 * self.T
        return (0, al(nt), al(nt) + al(nphi)), al(nt) + al(nphi) + al(nz)

    def _sample_views(self, buf):
        (ot, op, oz), _ = self._sample_layout()
        th = buf[ot:ot + 8 * self.D * self.K].view(torch.float64).view(self.D, self.K)
        ph = buf[op:op + 8 * self.K * self.V].view(torch.float64).view(self.K, self.V)
        z = buf[oz:oz + 4 * self.T].view(torch.int32)
        return th, ph, z

    def samples(self, n, first=1, every=1, stream=None):
        """Yields n samples (theta, phi, z) as host numpy arrays: the first
        after `first` sweeps, each further one `every` sweeps later.

        Each sample is packed into one of two alternating device snapshot
        buffers and copied, as one transfer, into a page-locked host buffer
        on a second stream, so the copy of sample i overlaps the sweeps that
        produce sample i + 1; the values are those state() would return at
        the same points (the three arrays of a sample share one host
        buffer)."""
        main = stream if stream is not None else torch.cuda.current_stream(self.dev)
        _, nbytes = self._sample_layout()
        if getattr(self, "_copy_stream", None) is None:
            self._copy_stream = torch.cuda.Stream(self.dev)
            self._snap = [torch.empty(nbytes, dtype=torch.uint8, device=self.dev) for _ in range(2)]
        cs = self._copy_stream
        copied = [None, None]
        pending = None
        for i in range(int(n)):
            self.sweep(first if i == 0 else every, stream=main)
            b = i & 1
            if copied[b] is not None:
                main.wait_event(copied[b])        # the copy out of this buffer is done
            th, ph, z = self._sample_views(self._snap[b])
            with torch.cuda.stream(main):
                th.copy_(self.theta)
                ph.copy_(self.phiT[:, :self.K].t())
                z.copy_(self.z)
                snap = torch.cuda.Event()
                snap.record(main)
            cs.wait_event(snap)
            with torch.cuda.stream(cs):
                host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
                host.copy_(self._snap[b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cs)
            copied[b] = ev
            if pending is not None:
                pending[1].synchronize()
                yield tuple(t.numpy() for t in self._sample_views(pending[0]))
            pending = (host, ev)
        if pending is not None:
            pending[1].synchronize()
            yield tuple(t.numpy() for t in self._sample_views(pending[0]))

    # ---- log densities -----------------------------------------------------
    def _ll_buffers(self):
        if getattr(self, "_ll_scratch", None) is None:
            self._ll_scratch = torch.zeros(int(N.lib().ab_ll_scratch_bytes()), dtype=torch.uint8, device=self.dev)
            self._ll_out = torch.zeros(1, dtype=torch.float64, device=self.dev)
        return self._ll_scratch, self._ll_out

    def ll_mod(self, stream=None):
        """The model log density of the current state, as the reference's
        augur_get_curr_ll returns it (its Dirichlet densities carry no
        normalising constant), computed on the device."""
        sc, out = self._ll_buffers()
        N.check(N.lib().ab_lda_ll_mod(self.D, self.K, self.V, N.ptr(self.doc_off), N.ptr(self.w), N.ptr(self.z),
                                      N.ptr(self.alpha), N.ptr(self.beta), N.ptr(self.theta), N.ptr(self.phiT),
                                      N.ptr(out), N.ptr(sc), N.stream_ptr(stream)), "ab_lda_ll_mod")
        return float(out.item())

    def pred_ll(self, w_heldout, stream=None):
        """Log-likelihood of held-out tokens under the current theta and phi:
        sum over tokens of log sum_k theta[d][k] phi[k][w] (the inner sum of
        experiments/lda/lda.py:149-173).  w_heldout: one token array per
        document (D of them), or a CSR pair (doc_off, w)."""
        if isinstance(w_heldout, tuple):
            off, w = (np.ascontiguousarray(a, np.int32) for a in w_heldout)
        else:
            off, w = flatten_docs(w_heldout)
        if len(off) != self.D + 1:
            raise ValueError("held-out tokens must be given for all %d documents" % self.D)
        if len(w) and (w.min() < 0 or w.max() >= self.V):
            raise ValueError("token ids must lie in [0, V)")
        sc, out = self._ll_buffers()
        off_d = torch.as_tensor(off).to(self.dev)
        w_d = torch.as_tensor(w).to(self.dev)
        N.check(N.lib().ab_lda_pred_ll(self.D, self.K, self.V, N.ptr(off_d), N.ptr(w_d), N.ptr(self.theta),
                                       N.ptr(self.phiT), N.ptr(out), N.ptr(sc), N.stream_ptr(stream)),
                "ab_lda_pred_ll")
        return float(out.item())

    # ---- sampling ----------------------------------------------------------
    @traced("lda.sweep")
    def sweep(self, n=1, graph=True, stream=None):
        N.check(N.lib().ab_lda_run(self._h, int(n), int(bool(graph)), N.stream_ptr(stream)),
                "ab_lda_run")
        self.iteration += int(n)

    def close(self):
        if getattr(self, "_h", None) is not None:
            N.lib().ab_lda_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def synthetic_corpus(K, V, D, mean_len, alpha, beta, seed):
    """Documents from the LDA generative process (numpy, seeded): lengths
    ~ Poisson(mean_len) (at least 1), theta ~ Dir(alpha), phi ~ Dir(beta)."""
    rng = np.random.default_rng(seed)
    lens = np.maximum(1, rng.poisson(mean_len, size=D)).astype(np.int64)
    theta = rng.dirichlet(np.full(K, alpha), size=D)
    phi = rng.dirichlet(np.full(V, beta), size=K)
    off = np.zeros(D + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    T = int(off[-1])
    doc_of = np.repeat(np.arange(D), lens)
    # z per token by inverse CDF on theta rows, then w by inverse CDF on phi rows
    u1, u2 = rng.random(T), rng.random(T)
    ct = np.cumsum(theta, axis=1)
    z = np.minimum((ct[doc_of] < u1[:, None]).sum(1), K - 1)
    cp = np.cumsum(phi, axis=1)
    w = np.empty(T, np.int64)
    for k in range(K):
        m = z == k
        if m.any():
            w[m] = np.minimum(np.searchsorted(cp[k], u2[m]), V - 1)
    return off.astype(np.int32), w.astype(np.int32)
