"""Batched HLR sampling on the tensor cores: host side of ab_hlrb_*, ab_hmcb_*
and the gradient surrogate (ab_mlp_*, ab_sur_*).

Model (compiler/augur/test/hlr.rv with the coefficient prior fixed):
    theta[d] ~ Normal(0, var)  or  StudentT(nu, scale)      d < D
    y[n] ~ Bernoulli(sigmoid(dotprod(theta, x[n])))
C chains share one bf16 design matrix; each chain is one FP32 row of
`theta` [C, D].  `BatchedHmc` runs the reference's HMC transition
(cbits/augur_mcmclib.h:343-424) for all chains with the exact gradient;
`SurrogateHmc` runs the same transition with the leapfrog driven by a small
MLP trained online on (theta, exact gradient) pairs that the sampler itself
produces, while the exact log density decides every accept.
"""
import ctypes as C
import math

import numpy as np
import torch

from . import _native as N
from .checkpoint import Checkpointable
from .trace import traced

PRIOR_NORMAL, PRIOR_STUDENT_T = 0, 1


class HlrbModelC(C.Structure):
    _fields_ = [("N", C.c_int), ("D", C.c_int), ("ldx", C.c_int), ("X", C.c_void_p), ("Xt", C.c_void_p),
                ("y", C.c_void_p), ("prior", C.c_int), ("prior_a", C.c_double), ("prior_b", C.c_double)]


class HmcbStateC(C.Structure):
    _fields_ = [("C", C.c_int), ("D", C.c_int), ("seed", C.c_ulonglong), ("iter", C.c_void_p),
                ("eps0", C.c_void_p), ("jitter", C.c_float), ("theta", C.c_void_p), ("p", C.c_void_p),
                ("g_cur", C.c_void_p), ("logp_cur", C.c_void_p), ("theta0", C.c_void_p), ("g0", C.c_void_p),
                ("logp0", C.c_void_p), ("H0", C.c_void_p), ("eps_c", C.c_void_p), ("stats", C.c_void_p)]


class MlpDescC(C.Structure):
    _fields_ = [("d_in", C.c_int), ("h1", C.c_int), ("h2", C.c_int), ("d_out", C.c_int), ("w", C.c_void_p),
                ("wb", C.c_void_p)]


class HlrbData:
    """Design matrix (bf16, device), its transpose, labels and the prior."""

    def __init__(self, X, y, prior="student_t", nu=3.0, scale=1.0, var=1.0, device="cuda"):
        X = torch.as_tensor(X)
        if X.dtype != torch.bfloat16:
            X = X.to(torch.float32).to(torch.bfloat16)
        self.X = X.to(device).contiguous()
        self.N, self.D = self.X.shape
        if self.D % 8:
            raise ValueError("D must be a multiple of 8 (16-byte rows for the tensor maps)")
        self.y = torch.as_tensor(y).to(device=device, dtype=torch.int32).contiguous()
        n_xt = int(N.lib().ab_hlrb_xt_elems(self.N, self.D))
        self.Xt = torch.empty(n_xt, dtype=torch.bfloat16, device=device)
        N.check(N.lib().ab_hlrb_transpose(self.N, self.D, N.ptr(self.X), self.D, N.ptr(self.Xt), N.stream_ptr()),
                "ab_hlrb_transpose")
        if prior == "student_t":
            self.prior, self.pa, self.pb = PRIOR_STUDENT_T, float(nu), float(scale)
        elif prior == "normal":
            self.prior, self.pa, self.pb = PRIOR_NORMAL, float(var), 0.0
        else:
            raise ValueError("prior must be 'student_t' or 'normal'")
        self.c = HlrbModelC(self.N, self.D, self.D, self.X.data_ptr(), self.Xt.data_ptr(), self.y.data_ptr(),
                            self.prior, self.pa, self.pb)
        self.device = self.X.device
        self.config = None     # ab_hlrb_config chosen by autotune(); None: built-in shapes

    def workspace(self, C_, config=None):
        """Device workspace for C_ chains under a launch shape (default: the
        shape chosen by autotune(), else the built-in one)."""
        cfg = self.config if config is None else config
        nb = int(N.lib().ab_hlrb_workspace_bytes_cfg(self.N, self.D, C_, C.byref(cfg) if cfg is not None else None))
        if nb == 0:
            raise N.AugurError("ab_hlrb_workspace_bytes_cfg: bad sizes or launch shape")
        return torch.empty(nb, dtype=torch.uint8, device=self.device)

    def autotune(self, C_, grad=True, tuner=None):
        """Time the candidate launch shapes of the pass for C_ chains on this
        GPU (augurv2_b200.autotune) and use the fastest from now on.  Call it
        before creating samplers: their workspaces are sized for the shape in
        force when they are made."""
        from . import autotune as T
        tuner = tuner or T.default_tuner()
        self.config = T.HlrbConfigC.of(tuner.hlrb(self, C_, grad))
        return self.config.as_dict()

    def logp_grad(self, theta, grad=True, logp_out=None, grad_out=None, work=None, err=None, stream=None,
                  logp=True, config=None):
        """(logp [C] f64 or None, grad [C, D] f32 or None) at theta [C, D] f32
        (device); logp=False skips the log-likelihood terms.  `config` (an
        autotune.HlrbConfigC) overrides the launch shape for this call; the
        workspace must have been sized for the same shape."""
        C_ = theta.shape[0]
        if not (grad or logp):
            raise ValueError("nothing to compute")
        cfg = self.config if config is None else config
        if logp and logp_out is None:
            logp_out = torch.empty(C_, dtype=torch.float64, device=self.device)
        if grad and grad_out is None:
            grad_out = torch.empty((C_, self.D), dtype=torch.float32, device=self.device)
        if work is None:
            work = self.workspace(C_, cfg)
        need = int(N.lib().ab_hlrb_workspace_bytes_cfg(self.N, self.D, C_, C.byref(cfg) if cfg is not None else None))
        if work.numel() * work.element_size() < need:
            raise N.AugurError("hlrb workspace holds %d bytes, this launch shape needs %d"
                               % (work.numel() * work.element_size(), need))
        N.check(N.lib().ab_hlrb_logp_grad_cfg(C.byref(self.c), C_, N.ptr(theta), theta.stride(0),
                                              N.ptr(logp_out) if logp else None,
                                              N.ptr(grad_out) if grad else None, self.D,
                                              C.byref(cfg) if cfg is not None else None, N.ptr(work),
                                              N.ptr(err) if err is not None else None, N.stream_ptr(stream)),
                "ab_hlrb_logp_grad_cfg")
        return (logp_out if logp else None), (grad_out if grad else None)


def synthetic(N_, D, seed=0, nu=3.0, device="cuda", chunk=1 << 18):
    """X ~ N(0,1) (bf16), beta ~ StudentT(nu), y ~ Bernoulli(sigmoid(X beta))."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    rs = np.random.default_rng(seed)
    beta = rs.standard_t(nu, size=D).astype(np.float32)
    X = torch.empty((N_, D), dtype=torch.bfloat16, device=device)
    y = torch.empty(N_, dtype=torch.int32, device=device)
    bt = torch.as_tensor(beta, device=device)
    for s in range(0, N_, chunk):
        e = min(N_, s + chunk)
        xs = torch.randn((e - s, D), generator=g, device=device)
        X[s:e] = xs.to(torch.bfloat16)
        t = X[s:e].float() @ bt
        y[s:e] = (torch.rand(e - s, generator=g, device=device) < torch.sigmoid(t)).to(torch.int32)
    return X, y, beta


class _ChainState:
    """Device buffers of ab_hmcb_state."""

    def __init__(self, C_, D, seed, eps, jitter, init, device):
        f32, f64 = torch.float32, torch.float64
        self.C, self.D = C_, D
        self.theta = torch.as_tensor(np.asarray(init, np.float32)).to(device).reshape(C_, D).contiguous()
        z = lambda *s, dt=f32: torch.zeros(*s, dtype=dt, device=device)
        self.p, self.g_cur, self.theta0, self.g0 = z(C_, D), z(C_, D), z(C_, D), z(C_, D)
        self.logp_cur, self.logp0, self.H0 = z(C_, dt=f64), z(C_, dt=f64), z(C_, dt=f64)
        self.eps_c = z(C_)
        self.stats = z(C_, 3, dt=f64)     # accepts, summed accept probability, divergences
        self.iter = torch.zeros(1, dtype=torch.int64, device=device)
        self.eps0 = torch.full((1,), float(eps), dtype=f32, device=device)
        self.c = HmcbStateC(C_, D, int(seed), self.iter.data_ptr(), self.eps0.data_ptr(), float(jitter),
                            self.theta.data_ptr(), self.p.data_ptr(), self.g_cur.data_ptr(),
                            self.logp_cur.data_ptr(), self.theta0.data_ptr(), self.g0.data_ptr(),
                            self.logp0.data_ptr(), self.H0.data_ptr(), self.eps_c.data_ptr(), self.stats.data_ptr())

    def begin(self, stream=None):
        N.check(N.lib().ab_hmcb_begin(C.byref(self.c), N.stream_ptr(stream)), "ab_hmcb_begin")

    def step(self, g, stream=None):
        N.check(N.lib().ab_hmcb_step(C.byref(self.c), N.ptr(g), N.stream_ptr(stream)), "ab_hmcb_step")

    def final(self, g_new, logp_new, stream=None):
        N.check(N.lib().ab_hmcb_final(C.byref(self.c), N.ptr(g_new), N.ptr(logp_new), N.stream_ptr(stream)),
                "ab_hmcb_final")


_CHAIN_TENSORS = ("s.theta", "s.p", "s.g_cur", "s.logp_cur", "s.theta0", "s.g0", "s.logp0", "s.H0", "s.eps_c", "s.stats", "s.iter", "s.eps0")


class BatchedHmc(Checkpointable):
    _ckpt_tensors = _CHAIN_TENSORS
    _ckpt_scalars = ("n_grad",)

    """C chains of exact-gradient HMC on an HlrbData: L leapfrog steps of size
    eps (jittered per chain by +-jitter), FP64 energies, one exact log density
    and gradient per step."""

    def __init__(self, data, C_, L=10, eps=0.01, jitter=0.1, seed=0, init=None):
        self.data, self.C, self.L = data, int(C_), int(L)
        D = data.D
        if init is None:
            init = np.zeros((self.C, D), np.float32)
        init = np.broadcast_to(np.asarray(init, np.float32), (self.C, D)).copy()
        self.s = _ChainState(self.C, D, seed, eps, jitter, init, data.device)
        self.work = data.workspace(self.C)
        self.err = torch.zeros(1, dtype=torch.int32, device=data.device)
        self.logp_new = torch.zeros(self.C, dtype=torch.float64, device=data.device)
        self.g_new = torch.zeros((self.C, D), dtype=torch.float32, device=data.device)
        self.n_grad = 0
        data.logp_grad(self.s.theta, True, self.s.logp_cur, self.s.g_cur, self.work, self.err)
        self.graph = None

    @property
    def theta(self):
        return self.s.theta

    def set_eps(self, eps):
        self.s.eps0.fill_(float(eps))

    def _iteration(self, stream=None):
        s, d = self.s, self.data
        s.begin(stream)
        for l in range(self.L):
            last = l == self.L - 1
            # the log density is needed only at the end point
            d.logp_grad(s.theta, True, self.logp_new, self.g_new, self.work, self.err, stream, logp=last)
            if not last:
                s.step(self.g_new, stream)
        s.final(self.g_new, self.logp_new, stream)

    def capture(self):
        """Capture one iteration (L exact passes) as a CUDA graph; the chain
        state is left as it was."""
        keep = (self.s.theta, self.s.g_cur, self.s.logp_cur, self.s.stats, self.s.iter)
        saved = [t.clone() for t in keep]
        side = torch.cuda.Stream(device=self.data.device)
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self._iteration(side)          # warm-up launch outside capture
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._iteration(torch.cuda.current_stream())
        for t, v in zip(keep, saved):
            t.copy_(v)

    @traced("hmcb.run")
    def run(self, n=1, record=None):
        for _ in range(int(n)):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._iteration()
            self.n_grad += self.L
            if record is not None:
                record.append(self.s.theta.clone())

    def accept_rate(self):
        st = self.s.stats.cpu().numpy()
        it = int(self.s.iter.item()) - getattr(self, "_iter0", 0)
        return st[:, 0].sum() / max(1, it * self.C), st[:, 1].sum() / max(1, it * self.C)

    def divergences(self):
        """Divergent transitions (energy error above AB_DIVERGENCE_DH, or not
        finite) summed over chains since the last reset_stats."""
        return int(self.s.stats[:, 2].sum().item())

    def reset_stats(self):
        """Restart the accept statistics (the iteration counter, which
        addresses the random streams, keeps counting)."""
        self.s.stats.zero_()
        self._iter0 = int(self.s.iter.item())


class MlpSurrogate(Checkpointable):
    _ckpt_tensors = ("w", "wb", "m", "v", "mu", "inv_s", "a", "h", "o", "M", "buf_theta", "buf_grad")
    _ckpt_scalars = ("step_count", "n_buf", "pos", "use_net", "dense")

    def _ckpt_extra(self):
        return {"gen": self.gen.get_state()}

    def _ckpt_load_extra(self, extra):
        self.gen.set_state(extra["gen"])

    """Gradient surrogate g(theta) ~ a + (theta - mu) M + o * MLP((theta - mu) / s).

    The linear part is a least-squares fit of the gradient on the parameters
    over the replay buffer: a dense D x D matrix M once the buffer holds at
    least 2 D pairs (the posterior's Hessian on average, so the surrogate's
    force field carries the posterior's correlations), a per-coordinate slope
    h before that.  The MLP d-h1-h2-d (GELU, bf16 weights, FP32 accumulation)
    learns the rest in units of the residual's per-coordinate scale o.
    Trained by Adam on (theta, gradient) pairs from the replay buffer."""

    def __init__(self, D, h1=256, h2=256, seed=0, device="cuda", capacity=8192, batch=512, lr=1e-3,
                 dense_linear=True):
        self.D, self.h1, self.h2 = D, h1, h2
        self.dense_linear = bool(dense_linear)   # False: per-coordinate slopes only
        self.device = device
        n = int(N.lib().ab_mlp_param_count(D, h1, h2, D))
        rs = np.random.default_rng(seed)
        w = np.zeros(n, np.float32)
        off = 0
        for fan_in, fan_out in ((D, h1), (h1, h2), (h2, D)):
            lim = math.sqrt(6.0 / (fan_in + fan_out))
            w[off:off + fan_in * fan_out] = rs.uniform(-lim, lim, fan_in * fan_out)
            off += fan_in * fan_out + fan_out
        # last layer starts at zero output: the surrogate begins as the linear fit
        w3 = n - D - h2 * D
        w[w3:w3 + h2 * D] *= 0.1
        self.w = torch.as_tensor(w).to(device)
        self.wb = torch.empty(n, dtype=torch.bfloat16, device=device)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.gw = torch.zeros_like(self.w)
        self.desc = MlpDescC(D, h1, h2, D, self.w.data_ptr(), self.wb.data_ptr())
        N.check(N.lib().ab_mlp_sync_bf16(C.byref(self.desc), N.stream_ptr()), "ab_mlp_sync_bf16")
        self.step_count = 0
        self.lr, self.batch = lr, int(batch)
        f = lambda: torch.zeros(D, dtype=torch.float32, device=device)
        self.mu, self.inv_s, self.a, self.h, self.o = f(), f() + 1.0, f(), f(), f() + 1.0
        self.M = torch.zeros((D, D), dtype=torch.float32, device=device)
        self.dense = False
        self.cap = int(capacity)
        self.buf_theta = torch.zeros((self.cap, D), dtype=torch.float32, device=device)
        self.buf_grad = torch.zeros((self.cap, D), dtype=torch.float32, device=device)
        self.n_buf, self.pos = 0, 0
        self._bufs = {}
        self.gen = torch.Generator(device=device)
        self.gen.manual_seed(int(seed) + 1)
        self.use_net = True

    def _scratch(self, B):
        if B not in self._bufs:
            D, dev = self.D, self.device
            self._bufs[B] = dict(
                z=torch.empty((B, D), dtype=torch.float32, device=dev),
                out=torch.empty((B, D), dtype=torch.float32, device=dev),
                act=torch.empty(int(N.lib().ab_mlp_act_floats(B, self.h1, self.h2)), dtype=torch.float32,
                                device=dev),
                bsc=torch.empty(int(N.lib().ab_mlp_backward_scratch_floats(B, self.h1, self.h2)),
                                dtype=torch.float32, device=dev),
                dy=torch.empty((B, D), dtype=torch.float32, device=dev),
                dt=torch.empty((B, D), dtype=torch.float32, device=dev),
                tgt=torch.empty((B, D), dtype=torch.float32, device=dev),
                rsq=torch.empty(B, dtype=torch.float64, device=dev),
            )
        return self._bufs[B]

    def add(self, theta, grad):
        """Append pairs (rows of theta, grad) to the replay ring; rows with a
        non-finite value (from a trajectory a broken surrogate drove) are
        left out."""
        ok = torch.isfinite(theta).all(1) & torch.isfinite(grad).all(1)
        if not bool(ok.all()):
            theta, grad = theta[ok], grad[ok]
        n = theta.shape[0]
        if n == 0:
            return
        idx = (torch.arange(n, device=self.device) + self.pos) % self.cap
        self.buf_theta[idx] = theta
        self.buf_grad[idx] = grad
        self.pos = (self.pos + n) % self.cap
        self.n_buf = min(self.cap, self.n_buf + n)

    def refit(self):
        """Input scaling and the linear part from the replay buffer: dense
        least squares (binary64 normal equations with a small ridge) when the
        buffer holds at least 2 D pairs, per-coordinate slopes otherwise.  All
        tensors are updated in place (captured graphs read them)."""
        th, g = self.buf_theta[:self.n_buf], self.buf_grad[:self.n_buf]
        mu = th.mean(0)
        dt = th - mu
        var = (dt * dt).mean(0).clamp_min(1e-30)
        gm = g.mean(0)
        self.mu.copy_(mu)
        self.inv_s.copy_(var.rsqrt())
        self.a.copy_(gm)
        M = None
        if self.dense_linear and self.n_buf >= 2 * self.D:
            X = dt.double()
            Y = (g - gm).double()
            A = X.T @ X
            A += torch.eye(self.D, dtype=torch.float64, device=self.device) * (1e-9 * A.diagonal().mean())
            M, info = torch.linalg.solve_ex(A, X.T @ Y)
            if int(info.item()) != 0 or not bool(torch.isfinite(M).all()):
                M = None
        if M is not None:
            self.M.copy_(M)
            self.h.zero_()
            self.dense = True
            res = g - gm - dt @ self.M
        else:
            h = ((g - gm) * dt).mean(0) / var
            self.h.copy_(h)
            self.M.zero_()
            self.dense = False
            res = g - gm - h * dt
        self.o.copy_((res * res).mean(0).sqrt().clamp_min(1e-12))

    def predict(self, theta, out_grad, stream=None):
        B = theta.shape[0]
        L, st = N.lib(), N.stream_ptr(stream)
        if self.use_net:
            N.check(L.ab_sur_predict(C.byref(self.desc), B, N.ptr(theta), theta.stride(0), N.ptr(self.mu),
                                     N.ptr(self.inv_s), N.ptr(self.a), N.ptr(self.h), N.ptr(self.o),
                                     N.ptr(out_grad), out_grad.stride(0), st), "ab_sur_predict")
            self._add_dense(theta, out_grad, stream)
            return out_grad
        sc = self._scratch(B)
        N.check(L.ab_sur_pre(B, self.D, N.ptr(theta), N.ptr(self.mu), N.ptr(self.inv_s), N.ptr(sc["z"]), st),
                "ab_sur_pre")
        if self.use_net:
            N.check(L.ab_mlp_forward(C.byref(self.desc), B, N.ptr(sc["z"]), self.D, N.ptr(sc["out"]), self.D,
                                     N.ptr(sc["act"]), st), "ab_mlp_forward")
        else:
            sc["out"].zero_()
        N.check(L.ab_sur_post(B, self.D, N.ptr(theta), N.ptr(sc["out"]), N.ptr(self.mu), N.ptr(self.a),
                              N.ptr(self.h), N.ptr(self.o), N.ptr(out_grad), st), "ab_sur_post")
        self._add_dense(theta, out_grad, stream)
        return out_grad

    def _add_dense(self, theta, out_grad, stream=None):
        """out += (theta - mu) M, the dense linear part (a plain FP32 GEMM),
        when it is in use."""
        if not self.dense:
            return
        B = theta.shape[0]
        sc = self._scratch(B)
        st = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(st):
            torch.sub(theta, self.mu, out=sc["dt"])
            out_grad.addmm_(sc["dt"], self.M)

    def train(self, steps):
        """Adam steps on minibatches of the replay buffer; returns the last
        minibatch's mean squared error in output units.  The minibatches of
        all steps are gathered and standardised in one pass."""
        if self.n_buf == 0 or not self.use_net:
            return float("nan")
        steps = int(steps)
        B = min(self.batch, self.n_buf)
        sc = self._scratch(B)
        key = ("train", steps, B)
        if key not in self._bufs:
            self._bufs[key] = (torch.empty((steps * B, self.D), dtype=torch.float32, device=self.device),
                               torch.empty((steps * B, self.D), dtype=torch.float32, device=self.device))
        zs, ts = self._bufs[key]
        idx = torch.randint(0, self.n_buf, (steps * B,), generator=self.gen, device=self.device)
        dt = torch.index_select(self.buf_theta, 0, idx).sub_(self.mu)
        torch.mul(dt, self.inv_s, out=zs)
        g = torch.index_select(self.buf_grad, 0, idx)
        if self.dense:
            g.sub_(dt @ self.M)
        torch.div(g.sub_(self.a).sub_(dt.mul_(self.h)), self.o, out=ts)
        L, st = N.lib(), N.stream_ptr()
        esz = zs.element_size() * B * self.D
        for i in range(steps):
            zp, tp = zs.data_ptr() + i * esz, ts.data_ptr() + i * esz
            N.check(L.ab_mlp_forward(C.byref(self.desc), B, zp, self.D, N.ptr(sc["out"]), self.D,
                                     N.ptr(sc["act"]), st), "ab_mlp_forward")
            N.check(L.ab_mlp_mse(B, self.D, N.ptr(sc["out"]), self.D, tp, self.D, N.ptr(sc["dy"]),
                                 N.ptr(sc["rsq"]), st), "ab_mlp_mse")
            N.check(L.ab_mlp_backward(C.byref(self.desc), B, zp, self.D, N.ptr(sc["dy"]),
                                      N.ptr(sc["act"]), N.ptr(self.gw), N.ptr(sc["bsc"]), st), "ab_mlp_backward")
            self.step_count += 1
            N.check(L.ab_mlp_adam(C.byref(self.desc), N.ptr(self.gw), N.ptr(self.m), N.ptr(self.v),
                                  self.step_count, self.lr, 0.9, 0.999, 1e-8, st), "ab_mlp_adam")
        return float(sc["rsq"].sum().item()) / (B * self.D)

    def rel_error(self, theta, grad):
        """Relative error |g_hat - g| / |g| (Frobenius) on given pairs."""
        gh = torch.empty_like(grad)
        self.predict(theta, gh)
        return float(torch.linalg.vector_norm(gh - grad) / torch.linalg.vector_norm(grad).clamp_min(1e-30))


class SurrogateHmc(Checkpointable):
    _ckpt_tensors = _CHAIN_TENSORS + ("g_exact",)
    _ckpt_scalars = ("it", "fallback", "last_rel_err", "n_grad", "n_logp", "learn_iters")

    def _ckpt_extra(self):
        return {"sur": self.sur.state_dict()}

    def _ckpt_load_extra(self, extra):
        self.sur.load_state_dict(extra["sur"])

    """HMC whose leapfrog uses the surrogate gradient; the exact log density
    (tensor-core forward pass) decides every accept.  Every `train_every`
    iterations the exact gradient at the proposals is computed too: during
    the first `learn_iters` iterations (all of them when None) those pairs
    join the replay buffer, the surrogate's linear part is refitted and the
    network trained; at every such check the surrogate's relative error on
    the fresh pairs is measured, and above `max_rel_err` the sampler falls
    back to exact-gradient HMC until a later check passes.

    With a surrogate that no longer changes (after `learn_iters`), each
    iteration is a fixed HMC kernel with a position-only force and an exact
    Metropolis test, which leaves the posterior invariant; while the
    surrogate is still learning from the chains' own states the kernel
    adapts, which is why learning belongs to the warm-up.

    The fallback bound guards efficiency, not exactness (the accept test is
    exact whatever the force): a surrogate fitted with per-coordinate slopes
    only, at relative error 0.08 on the 2e6 x 512 problem, left the chains
    mixing about 60 times slower per iteration than exact-gradient HMC, while
    surrogates with the dense linear part measure 0.002 - 0.03 after their
    warm-up; 0.05 lies between."""

    def __init__(self, data, C_, L=10, eps=0.01, jitter=0.1, seed=0, init=None, surrogate=None,
                 train_every=4, train_steps=20, max_rel_err=0.05, learn_iters=None):
        self.data, self.C, self.L = data, int(C_), int(L)
        D = data.D
        if init is None:
            init = np.zeros((self.C, D), np.float32)
        init = np.broadcast_to(np.asarray(init, np.float32), (self.C, D)).copy()
        self.s = _ChainState(self.C, D, seed, eps, jitter, init, data.device)
        self.sur = surrogate if surrogate is not None else MlpSurrogate(D, seed=seed, device=data.device)
        self.work = data.workspace(self.C)
        self.err = torch.zeros(1, dtype=torch.int32, device=data.device)
        self.logp_new = torch.zeros(self.C, dtype=torch.float64, device=data.device)
        self.g_new = torch.zeros((self.C, D), dtype=torch.float32, device=data.device)
        self.g_exact = torch.zeros((self.C, D), dtype=torch.float32, device=data.device)
        self.train_every, self.train_steps, self.max_rel_err = int(train_every), int(train_steps), max_rel_err
        self.learn_iters = learn_iters
        self.n_grad = 0          # exact gradient passes (forward + backward)
        self.n_logp = 0          # exact log-density-only passes
        self.it = 0
        self.fallback = False
        self.last_rel_err = float("nan")
        data.logp_grad(self.s.theta, True, self.s.logp_cur, self.g_exact, self.work, self.err)
        self.n_grad += 1
        self.sur.add(self.s.theta, self.g_exact)
        self.sur.refit()
        self.sur.predict(self.s.theta, self.s.g_cur)

    @property
    def theta(self):
        return self.s.theta

    def set_eps(self, eps):
        self.s.eps0.fill_(float(eps))

    def _refresh_current(self):
        """After the surrogate changes, the gradient at the current points is
        re-evaluated so that every trajectory uses one force field."""
        if self.fallback:
            self.data.logp_grad(self.s.theta, True, self.s.logp_cur, self.s.g_cur, self.work, self.err)
            self.n_grad += 1
        else:
            self.sur.predict(self.s.theta, self.s.g_cur)

    def learning(self):
        """True while checks still train the surrogate (the warm-up)."""
        return self.learn_iters is None or self.it < self.learn_iters

    def iteration(self, learn=True):
        s, d = self.s, self.data
        check = learn and (self.it % self.train_every == 0)
        training = check and self.learning()
        s.begin()
        for l in range(self.L):
            last = l == self.L - 1
            if self.fallback or (last and check):
                d.logp_grad(s.theta, True, self.logp_new, self.g_exact, self.work, self.err, logp=last)
                self.n_grad += 1
                if self.fallback:
                    self.g_new.copy_(self.g_exact)
                else:
                    self.sur.predict(s.theta, self.g_new)
            elif last:
                d.logp_grad(s.theta, False, self.logp_new, None, self.work, self.err)
                self.n_logp += 1
                self.sur.predict(s.theta, self.g_new)
            else:
                self.sur.predict(s.theta, self.g_new)
            if not last:
                s.step(self.g_new)
        if check:
            # fresh exact pairs at the proposals: error check (and, while
            # learning, new training data)
            self.last_rel_err = self.sur.rel_error(s.theta, self.g_exact)
            if training:
                self.sur.add(s.theta, self.g_exact)
        s.final(self.g_new, self.logp_new)
        self.it += 1
        if check:
            was = self.fallback
            self.fallback = not (self.last_rel_err <= self.max_rel_err)
            if training:
                self.sur.refit()
                if self.train_steps > 0:
                    self.sur.train(self.train_steps)
            if training or was != self.fallback:
                self._refresh_current()

    def _plain_iteration(self, stream=None):
        """A surrogate trajectory without the exact gradient check."""
        s, d = self.s, self.data
        s.begin(stream)
        for l in range(self.L):
            if l == self.L - 1:
                d.logp_grad(s.theta, False, self.logp_new, None, self.work, self.err, stream)
            self.sur.predict(s.theta, self.g_new, stream)
            if l < self.L - 1:
                s.step(self.g_new, stream)
        s.final(self.g_new, self.logp_new, stream)

    def capture(self):
        """Capture a surrogate trajectory (no check, no training) as a CUDA graph."""
        side = torch.cuda.Stream(device=self.data.device)
        side.wait_stream(torch.cuda.current_stream())
        saved = [t.clone() for t in (self.s.theta, self.s.g_cur, self.s.logp_cur, self.s.stats, self.s.iter)]
        with torch.cuda.stream(side):
            self._plain_iteration(side)      # warm-up launch outside capture
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._plain_iteration(torch.cuda.current_stream())
        for t, v in zip((self.s.theta, self.s.g_cur, self.s.logp_cur, self.s.stats, self.s.iter), saved):
            t.copy_(v)

    @traced("surrogate.run")
    def run(self, n=1, learn=True, record=None):
        for _ in range(int(n)):
            check = learn and (self.it % self.train_every == 0)
            if (not check) and (not self.fallback) and getattr(self, "graph", None) is not None:
                self.graph.replay()
                self.n_logp += 1
                self.it += 1
            else:
                self.iteration(learn)
            if record is not None:
                record.append(self.s.theta.clone())

    def accept_rate(self):
        st = self.s.stats.cpu().numpy()
        it = int(self.s.iter.item()) - getattr(self, "_iter0", 0)
        return st[:, 0].sum() / max(1, it * self.C), st[:, 1].sum() / max(1, it * self.C)

    def divergences(self):
        """Divergent transitions (energy error above AB_DIVERGENCE_DH, or not
        finite) summed over chains since the last reset_stats."""
        return int(self.s.stats[:, 2].sum().item())

    def reset_stats(self):
        """Restart the accept statistics (the iteration counter, which
        addresses the random streams, keeps counting)."""
        self.s.stats.zero_()
        self._iter0 = int(self.s.iter.item())


def adapt_step_size(sampler, n, target=0.8, rate=1.5, lo=1e-6, hi=10.0, run_kw=None):
    """Warm-up: after each iteration multiply the base step size by
    exp(rate * (mean acceptance probability - target)).  Returns the final
    step size."""
    run_kw = run_kw or {}
    eps = float(sampler.s.eps0.item())
    for _ in range(int(n)):
        before = sampler.s.stats[:, 1].sum().item()
        sampler.run(1, **run_kw)
        a = (sampler.s.stats[:, 1].sum().item() - before) / sampler.C
        eps = float(min(hi, max(lo, eps * math.exp(rate * (a - target)))))
        sampler.set_eps(eps)
    return eps


class BatchedNuts(Checkpointable):
    # the resumable tree walks, draw histories and iteration counters
    _ckpt_tensors = ("mem", "logp_new", "g_new")
    _ckpt_scalars = ("rounds",)

    """C chains of the reference's NUTS (cbits/augur_mcmclib.h:575-776) on an
    HlrbData, advanced together: each round every chain walks its tree to the
    next leaf (ab_nutsb_advance) and one tensor-core pass evaluates the log
    density and gradient at all chains' leaf positions.  Chains restart as
    soon as their tree terminates, each recording its draws (up to
    `hist_cap`).  One round can be captured as a CUDA graph.

    variant="reference" selects each iteration's draw as the reference does
    (the last doubling's pick only, with the truncated acceptance ratio), so
    draws equal the reference sampler's; variant="standard" uses Hoffman &
    Gelman's rule (the latest accepted pick of any doubling, probability
    min(1, n'/n)), which moves the chain on far more iterations."""

    VARIANTS = {"reference": 0, "standard": 1}

    def __init__(self, data, C_, eps, max_depth=10, seed=0, init=None, hist_cap=256, comp=0, iter0=0,
                 variant="reference"):
        if variant not in self.VARIANTS:
            raise ValueError("variant must be 'reference' or 'standard'")
        self.variant = variant
        self.data, self.C, self.D = data, int(C_), data.D
        self.eps, self.max_depth, self.seed, self.comp = float(eps), int(max_depth), int(seed), int(comp)
        self.hist_cap = int(hist_cap)
        D, dev = self.D, data.device
        if init is None:
            init = np.zeros((self.C, D), np.float32)
        init = np.broadcast_to(np.asarray(init, np.float32), (self.C, D)).copy()
        nb = int(N.lib().ab_nutsb_state_bytes(self.C, D, self.hist_cap))
        self.mem = torch.zeros(nb, dtype=torch.uint8, device=dev)
        th = torch.as_tensor(init).to(dev).contiguous()
        self.work = data.workspace(self.C)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.logp_new = torch.zeros(self.C, dtype=torch.float64, device=dev)
        self.g_new = torch.zeros((self.C, D), dtype=torch.float32, device=dev)
        lp, g = data.logp_grad(th, True, work=self.work, err=self.err)
        N.check(N.lib().ab_nutsb_init(N.ptr(self.mem), self.C, D, self.hist_cap, N.ptr(th), N.ptr(g), N.ptr(lp),
                                      int(iter0), N.stream_ptr()), "ab_nutsb_init")
        pt, ph, pd = C.c_void_p(), C.c_void_p(), C.c_void_p()
        N.check(N.lib().ab_nutsb_thprop(N.ptr(self.mem), self.C, D, self.hist_cap, C.byref(pt), C.byref(ph),
                                        C.byref(pd)), "ab_nutsb_thprop")
        base = self.mem.data_ptr()
        f32 = self.mem.view(torch.float32) if nb % 4 == 0 else None
        off_t, off_h, off_d = pt.value - base, ph.value - base, pd.value - base
        self.thprop = self.mem[off_t:off_t + 4 * self.C * D].view(torch.float32).view(self.C, D)
        self.hist = self.mem[off_h:off_h + 4 * self.C * self.hist_cap * D].view(torch.float32).view(
            self.C, self.hist_cap, D)
        self.hist_depth = self.mem[off_d:off_d + 4 * self.C * self.hist_cap].view(torch.int32).view(
            self.C, self.hist_cap)
        self.info_buf = torch.zeros((self.C, 7), dtype=torch.float64, device=dev)
        self.rounds = 0
        self.graph = None
        del f32

    def _round(self, stream=None):
        N.check(N.lib().ab_nutsb_advance_variant(N.ptr(self.mem), self.C, self.D, self.hist_cap, self.max_depth,
                                                 self.eps, self.seed, self.comp, self.VARIANTS[self.variant],
                                                 N.ptr(self.logp_new), N.ptr(self.g_new), N.stream_ptr(stream)),
                "ab_nutsb_advance_variant")
        self.data.logp_grad(self.thprop, True, self.logp_new, self.g_new, self.work, self.err, stream)

    def capture(self, stream=None):
        """Capture one round (advance + pass) as a CUDA graph.  The capture
        itself does not run the round; a warm-up round runs first."""
        self._round(stream)
        self.rounds += 1
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=stream):
            self._round(torch.cuda.current_stream())

    @traced("nutsb.run")
    def run(self, rounds):
        for _ in range(int(rounds)):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._round()
            self.rounds += 1

    def reset_history(self, stream=None):
        """End of warm-up: forget the recorded draws, keep every chain's state."""
        N.check(N.lib().ab_nutsb_reset_history(N.ptr(self.mem), self.C, self.D, self.hist_cap,
                                               N.stream_ptr(stream)), "ab_nutsb_reset_history")

    def info(self):
        N.check(N.lib().ab_nutsb_info(N.ptr(self.mem), self.C, self.D, self.hist_cap, N.ptr(self.info_buf),
                                      N.stream_ptr()), "ab_nutsb_info")
        return self.info_buf.cpu().numpy()

    def divergences(self):
        """Divergent iterations (a leaf below the slice level by more than
        AB_DIVERGENCE_DH) summed over chains since the last reset_history."""
        return int(self.info()[:, 6].sum())

    def draws(self):
        """[n, C, D]: the first n draws of every chain, n = the smallest count."""
        inf = self.info()
        if np.any(inf[:, 3] != 0):
            raise N.AugurError("batched NUTS: a chain reported an error")
        n = int(min(inf[:, 0].min(), self.hist_cap))
        return self.hist[:, :n].permute(1, 0, 2).cpu().numpy()


def lpt_assign(costs, n_streams, keys=None):
    """Longest-processing-time-first assignment of jobs to streams: the
    costliest job goes to the least-loaded stream, and so on.  Returns
    {key: stream index} (keys default to 0..len(costs)-1)."""
    keys = list(range(len(costs))) if keys is None else list(keys)
    load = [0.0] * int(n_streams)
    out = {}
    for c, k in sorted(zip(costs, keys), key=lambda ck: -ck[0]):
        q = min(range(len(load)), key=lambda j: load[j])
        out[k] = q
        load[q] += c
    return out


class NutsPool:
    """Many BatchedNuts samplers of uneven cost (model instances with their
    own N and D) sharing one GPU.

    Each sampler's round (leaf advance + tensor-core pass) is a captured CUDA
    graph; rounds are replayed in blocks over a few streams, samplers
    assigned to streams longest-processing-time first on their cost per
    round and re-balanced every block among the samplers still running.
    Shares: by default every running sampler replays `block` rounds per
    block; with share="time" a sampler replays rounds in inverse proportion
    to its cost per round (N * D plus a fixed launch overhead, up to
    MAX_SHARE times the block).  A sampler stops once every one of its chains
    has `min_draws` draws (or its draw history is full, or it ran
    `max_rounds` rounds in this call); the pool returns when all have
    stopped."""

    OVERHEAD = 5.0e6      # fixed cost of a round (launch latency), in N * D units
    MAX_SHARE = 4         # a block gives a sampler at most this many times `block` rounds
                          # (bounds the host time spent enqueueing graph launches)

    def __init__(self, samplers, streams=8, costs=None):
        self.samplers = list(samplers)
        self.streams = [torch.cuda.Stream() for _ in range(int(streams))]
        self.costs = [float(c) for c in costs] if costs is not None else \
            [float(s.data.N) * float(s.data.D) + self.OVERHEAD for s in self.samplers]
        self.rounds = [0] * len(self.samplers)
        self.done = [False] * len(self.samplers)
        for i, s in enumerate(self.samplers):
            if s.graph is None:
                st = self.streams[i % len(self.streams)]
                with torch.cuda.stream(st):
                    s.capture(st)
                self.rounds[i] = s.rounds
        torch.cuda.synchronize()

    def _assign(self, active, reps):
        return lpt_assign([self.costs[i] * reps[i] for i in active], len(self.streams), keys=active)

    def reset(self):
        """Start a new phase: every sampler runs again and its recorded draws
        are forgotten (the chains keep their states)."""
        for s in self.samplers:
            s.reset_history()
        self.done = [False] * len(self.samplers)

    def draws(self, i):
        """Draws recorded by sampler i's slowest chain."""
        return int(self.samplers[i].info()[:, 0].min())

    @traced("nuts_pool.run")
    def run(self, min_draws, max_rounds, block=25, share="equal"):
        """Replay rounds until every sampler has min_draws draws per chain;
        returns the number of rounds each sampler ran in this call.  share:
        "equal" (block rounds each per block) or "time" (rounds per block in
        inverse proportion to cost: cheap samplers keep drawing while the
        expensive ones finish, at the price of competing with them)."""
        cur = torch.cuda.current_stream()
        start = list(self.rounds)
        ran = lambda i: self.rounds[i] - start[i]
        cmax = max(self.costs) if self.costs else 1.0
        counts = [0] * len(self.samplers)
        self.done = [False] * len(self.samplers)
        while True:
            active = [i for i, d in enumerate(self.done) if not d]
            if not active:
                break
            reps = {i: (block if share == "equal" else
                        max(1, min(self.MAX_SHARE * block, int(round(block * cmax / self.costs[i])))))
                    for i in active}
            reps = {i: max(0, min(r, max_rounds - ran(i))) for i, r in reps.items()}
            where = self._assign(active, reps)
            for st in self.streams:
                st.wait_stream(cur)
            for i in active:
                with torch.cuda.stream(self.streams[where[i]]):
                    for _ in range(reps[i]):
                        self.samplers[i].graph.replay()
                self.rounds[i] += reps[i]
            for st in self.streams:
                cur.wait_stream(st)
            for i in active:
                s = self.samplers[i]
                s.rounds = self.rounds[i]
                counts[i] = self.draws(i)
                if ran(i) >= max_rounds or counts[i] >= min(min_draws, s.hist_cap):
                    self.done[i] = True
        return [ran(i) for i in range(len(self.samplers))]


class NutsgInstC(C.Structure):
    _fields_ = [("state", C.c_void_p), ("C", C.c_int), ("P", C.c_int), ("hist_cap", C.c_int),
                ("max_depth", C.c_int), ("variant", C.c_int), ("eps", C.c_double), ("seed", C.c_uint64),
                ("comp", C.c_uint32), ("logp_new", C.c_void_p), ("g_new", C.c_void_p)]


class HlrGroup:
    """Log density and gradient of many HlrbData instances, each with its own
    chains, with one launch per stage (ab_hlrg_*): when every D <= 256 the
    fused tensor-core kernel (forward, residual and backward per 128-row
    tile, the residual kept on chip, the work units of all instances on one
    persistent grid); otherwise the two-GEMM pass over all instances' tiles.
    Bind each instance's theta [C_i, D_i] f32 and logp [C_i] f64 / grad
    [C_i, D_i] f32 outputs (device tensors that outlive the group), then
    choose the active instances; the tables live in device memory, so a CUDA
    graph captured around logp_grad() follows later set_active() calls."""

    def __init__(self, datas, chains):
        L = N.lib()
        self.datas = list(datas)
        n = len(self.datas)
        if n == 0:
            raise ValueError("HlrGroup needs at least one data set")
        models = (HlrbModelC * n)(*[d.c for d in self.datas])
        cs = (C.c_int * n)(*[int(c) for c in chains])
        self._h = C.c_void_p()
        N.check(L.ab_hlrg_create(n, models, cs, C.byref(self._h)), "ab_hlrg_create")
        self.fused = bool(L.ab_hlrg_fused(self._h))

    def bind(self, i, theta, logp, grad):
        N.check(N.lib().ab_hlrg_bind(self._h, i, N.ptr(theta), theta.stride(0), N.ptr(logp), N.ptr(grad),
                                     grad.stride(0)), "ab_hlrg_bind")

    def set_active(self, active, stream=None):
        a = (C.c_int * len(self.datas))(*[1 if x else 0 for x in active])
        N.check(N.lib().ab_hlrg_set_active(self._h, a, N.stream_ptr(stream)), "ab_hlrg_set_active")

    def logp_grad(self, err=None, stream=None):
        N.check(N.lib().ab_hlrg_logp_grad(self._h, N.ptr(err) if err is not None else None, N.stream_ptr(stream)),
                "ab_hlrg_logp_grad")

    def close(self):
        if getattr(self, "_h", None):
            N.lib().ab_hlrg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NutsGroup:
    """Many BatchedNuts samplers of uneven size (model instances with their
    own N and D) advanced together with ONE launch per stage: a round is one
    grouped advance launch (every running instance's chains walk to their
    next leaf, ab_nutsg_advance) and one HlrGroup pass over all of their
    data sets (theta split, the fused tensor-core kernel, finishing sums),
    captured as one CUDA graph.  An instance's results are the same alone or
    in any group.  An instance leaves the launches once every one of its
    chains has `min_draws` draws (or its history is full, or it ran
    `max_rounds` rounds in this call); the instance tables live in device
    memory, so the captured graph follows the shrinking set without being
    captured again."""

    def __init__(self, samplers):
        L = N.lib()
        self.samplers = list(samplers)
        n = len(self.samplers)
        if n == 0:
            raise ValueError("NutsGroup needs at least one sampler")
        dev = self.samplers[0].data.device
        self._pass = HlrGroup([s.data for s in self.samplers], [s.C for s in self.samplers])
        self._adv = C.c_void_p()
        try:
            for i, s in enumerate(self.samplers):
                self._pass.bind(i, s.thprop, s.logp_new, s.g_new)
            insts = (NutsgInstC * n)(*[NutsgInstC(s.mem.data_ptr(), s.C, s.D, s.hist_cap, s.max_depth,
                                                  BatchedNuts.VARIANTS[s.variant], s.eps, s.seed, s.comp,
                                                  s.logp_new.data_ptr(), s.g_new.data_ptr())
                                       for s in self.samplers])
            N.check(L.ab_nutsg_create(n, insts, C.byref(self._adv)), "ab_nutsg_create")
        except Exception:
            self.close()
            raise
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.draw_buf = torch.zeros(2 * n, dtype=torch.int32, device=dev)
        self.active = [True] * n
        self.rounds = [s.rounds for s in self.samplers]
        self.graph = None
        self._set_active(self.active)

    def _set_active(self, active, stream=None):
        n = len(self.samplers)
        a = (C.c_int * n)(*[1 if x else 0 for x in active])
        self._pass.set_active(active, stream)
        N.check(N.lib().ab_nutsg_set_active(self._adv, a, N.stream_ptr(stream)), "ab_nutsg_set_active")
        self.active = list(active)

    def _round(self, stream=None):
        N.check(N.lib().ab_nutsg_advance(self._adv, N.stream_ptr(stream)), "ab_nutsg_advance")
        self._pass.logp_grad(self.err, stream)

    def _count(self, reps):
        for i, a in enumerate(self.active):
            if a:
                self.rounds[i] += reps
                self.samplers[i].rounds = self.rounds[i]

    def capture(self):
        """Run one round, then capture a round as a CUDA graph."""
        self._round()
        self._count(1)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._round(torch.cuda.current_stream())

    def step(self, rounds=1):
        """`rounds` rounds of every active instance."""
        for _ in range(int(rounds)):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._round()
        self._count(int(rounds))

    def min_draws(self):
        """[n] smallest draw count over each instance's chains (raises if a
        chain reported an error or the pass timed out)."""
        N.check(N.lib().ab_nutsg_min_draws(self._adv, N.ptr(self.draw_buf), N.stream_ptr()), "ab_nutsg_min_draws")
        d = self.draw_buf.cpu().numpy().reshape(-1, 2)
        if d[:, 1].any() or int(self.err.item()):
            raise N.AugurError("grouped NUTS: a chain reported an error or the pass timed out")
        return d[:, 0]

    def reset(self):
        """Start a new phase: every instance runs again and its recorded
        draws are forgotten (the chains keep their states)."""
        for s in self.samplers:
            s.reset_history()
        self._set_active([True] * len(self.samplers))

    def _rounds_to_first_finish(self, d, ran, min_draws):
        """Rounds until the first active instance is expected to reach its
        draw target, from the draws per round its slowest chain made so far
        in this call (at least 1; None before any instance has drawn)."""
        best = None
        for i, a in enumerate(self.active):
            r = ran(i)
            if not a or r <= 0 or d[i] <= 0:
                continue
            target = min(min_draws, self.samplers[i].hist_cap)
            est = -(-(target - int(d[i])) * r // int(d[i]))      # ceil
            best = est if best is None else min(best, est)
        return None if best is None else max(1, best)

    @traced("nuts_group.run")
    def run(self, min_draws, max_rounds, block=25):
        """Rounds until every instance has min_draws draws per chain; returns
        the rounds each instance ran in this call.  The draw counts are read
        back every `block` rounds, or sooner when an instance is expected to
        reach its target earlier (so that a large instance does not run up to
        `block` rounds past its target; each read-back is one host round trip)."""
        start = list(self.rounds)
        ran = lambda i: self.rounds[i] - start[i]
        if self.graph is None:
            self.capture()
        self._set_active([True] * len(self.samplers))
        d = None
        while any(self.active):
            reps = min(block, min(max_rounds - ran(i) for i, a in enumerate(self.active) if a))
            if d is not None:
                est = self._rounds_to_first_finish(d, ran, min_draws)
                if est is not None:
                    reps = min(reps, est)
            if reps > 0:
                self.step(reps)
            d = self.min_draws()
            act = [a and not (ran(i) >= max_rounds or d[i] >= min(min_draws, self.samplers[i].hist_cap))
                   for i, a in enumerate(self.active)]
            if act != self.active:
                self._set_active(act)
        return [ran(i) for i in range(len(self.samplers))]

    def close(self):
        self.graph = None
        if getattr(self, "_adv", None):
            N.lib().ab_nutsg_destroy(self._adv)
            self._adv = None
        if getattr(self, "_pass", None):
            self._pass.close()
            self._pass = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
