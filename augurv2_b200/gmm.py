"""Gaussian-mixture Gibbs samplers on the GPU: host side of ab_gmm_*.

Models (compiler/augur/test):
  mvgmm.rv   mu[k] ~ MvNormal(mu0, covs0); z[n] ~ Categorical(pis);
             y[n] ~ MvNormal(mu[z[n]], covs)                 (pis, covs fixed)
  hmvgmm.rv  pis ~ Dirichlet(alpha); mu[k] ~ MvNormal(mu0, covs0);
             cov[k] ~ InvWishart(df, scale0); z[n] ~ Categorical(pis);
             y[n] ~ MvNormal(mu[z[n]], cov[z[n]])
Schedules: ConjGibbs over the continuous parameters (in model order) then
DiscGibbs [z]; for mvgmm also ESlice [mu] or MWG [mu] ~ MvNormal(mu[k], S)
in place of ConjGibbs [mu].  Every kernel runs on the device (gmm.cu).
"""
import ctypes as C

import numpy as np
import torch

from . import _native as N
from .checkpoint import Checkpointable
from .trace import traced


class GmmGibbs(Checkpointable):
    _ckpt_tensors = ("mu", "cov", "pis", "z", "Linv", "hdet", "cnt", "sum", "obs", "shrinks", "accepts")
    _ckpt_scalars = ("iteration", "seed")

    def __init__(self, Y, K, mu0, cov0, pis=None, covs=None, alpha=None, df=None, scale0=None,
                 mu=None, cov=None, z=None, move="conj", prop_cov=None, compat=True, seed=0, iter0=0,
                 device="cuda"):
        """Shared-covariance mvgmm when `covs` is given, else hmvgmm."""
        Y = np.asarray(Y)
        self.N, self.d = Y.shape
        self.K = int(K)
        self.shared = covs is not None
        self.move = move
        self.seed, self.iteration, self.compat = int(seed), int(iter0), bool(compat)
        d, K = self.d, self.K
        dev = torch.device(device)
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64)).to(dev)
        self.Y = torch.as_tensor(np.ascontiguousarray(Y, np.float32)).to(dev)
        self.mu0, self.cov0 = f64(np.broadcast_to(mu0, (d,)).copy()), f64(cov0)
        if self.shared:
            self.pis = f64(pis if pis is not None else np.full(K, 1.0 / K))
            self.cov = f64(np.asarray(covs).reshape(1, d, d))
            if move != "conj":
                assert move in ("eslice", "mwg")
        else:
            assert move == "conj", "hmvgmm supports the conjugate schedule"
            self.alpha = f64(alpha if alpha is not None else np.ones(K))
            self.df = int(df if df is not None else d + 2)
            self.scale0 = f64(scale0 if scale0 is not None else np.eye(d))
            self.pis = f64(pis if pis is not None else np.full(K, 1.0 / K))
            self.cov = f64(cov if cov is not None else np.broadcast_to(np.eye(d), (K, d, d)).copy())
        self.mu = f64(mu if mu is not None else np.zeros((K, d)))
        self.z = torch.as_tensor(np.ascontiguousarray(z if z is not None else np.zeros(self.N), np.int32)).to(dev)
        self.prop_cov = f64(prop_cov if prop_cov is not None else cov0)
        Kc = 1 if self.shared else K
        self.Kc = Kc
        # tables: component slots [0, Kc), prior slot Kc, proposal slot Kc + 1,
        # inverse-Wishart scale slot Kc + 2 (hmvgmm)
        self.Linv = torch.zeros((Kc + 3, d, d), dtype=torch.float64, device=dev)
        self.hdet = torch.zeros(Kc + 3, dtype=torch.float64, device=dev)
        self.cnt = torch.zeros(K, dtype=torch.int32, device=dev)
        self.sum = torch.zeros((K, d), dtype=torch.float64, device=dev)
        self.obs = torch.zeros((K, d, d), dtype=torch.float64, device=dev)
        self.chi = torch.zeros((K, d), dtype=torch.float64, device=dev)     # Bartlett chi-square sums
        self._side = None
        self.scratch = torch.zeros(int(N.lib().ab_gmm_stats_scratch_bytes(d, K)) // 8 + 1,
                                   dtype=torch.float64, device=dev)
        # the screened assignment draw's tables and queue (ab_gmm_disc_z_screened)
        self.zscratch = torch.zeros(int(N.lib().ab_gmm_z_scratch_bytes(self.N, d, K)), dtype=torch.uint8,
                                    device=dev)
        self.shrinks = torch.zeros(K, dtype=torch.int32, device=dev)
        self.accepts = torch.zeros(K, dtype=torch.int32, device=dev)
        L = N.lib()
        st = N.stream_ptr()
        N.check(L.ab_gmm_prep(1, d, N.ptr(self.cov0), N.ptr(self.Linv[Kc]), N.ptr(self.hdet[Kc:]), st), "prep")
        N.check(L.ab_gmm_prep(1, d, N.ptr(self.prop_cov), N.ptr(self.Linv[Kc + 1]), N.ptr(self.hdet[Kc + 1:]), st),
                "prep")
        if self.shared:
            N.check(L.ab_gmm_prep(1, d, N.ptr(self.cov), N.ptr(self.Linv), N.ptr(self.hdet), st), "prep")
        else:
            N.check(L.ab_gmm_prep(1, d, N.ptr(self.scale0), N.ptr(self.Linv[Kc + 2]), N.ptr(self.hdet[Kc + 2:]),
                                  st), "prep")

    # ---- log densities -----------------------------------------------------
    def _ll_buffers(self):
        if getattr(self, "_ll_scratch", None) is None:
            dev = self.Y.device
            self._ll_scratch = torch.zeros(int(N.lib().ab_ll_scratch_bytes()), dtype=torch.uint8, device=dev)
            self._ll_out = torch.zeros(1, dtype=torch.float64, device=dev)
        return self._ll_scratch, self._ll_out

    def _refresh_tables(self, st):
        if not self.shared:     # the component tables of the current covariances
            N.check(N.lib().ab_gmm_prep(self.K, self.d, N.ptr(self.cov), N.ptr(self.Linv), N.ptr(self.hdet), st),
                    "prep")

    def ll_mod(self, stream=None):
        """The model log density of the current state, as the reference's
        augur_get_curr_ll returns it (hmvgmm.rv or mvgmm.rv: Dirichlet
        weights without normalising constant, normal means, inverse-Wishart
        covariances, categorical labels, normal data), on the device."""
        st = N.stream_ptr(stream)
        self._refresh_tables(st)
        sc, out = self._ll_buffers()
        Kc = self.Kc
        N.check(N.lib().ab_gmm_ll_mod(
            self.N, self.d, self.K, int(self.shared), N.ptr(self.Y), N.ptr(self.z), N.ptr(self.pis), N.ptr(self.mu),
            N.ptr(self.Linv), N.ptr(self.hdet), N.ptr(self.mu0), N.ptr(self.Linv[Kc]), N.ptr(self.hdet[Kc:]),
            None if self.shared else N.ptr(self.alpha), 0 if self.shared else self.df,
            None if self.shared else N.ptr(self.scale0), None if self.shared else N.ptr(self.hdet[Kc + 2:]),
            N.ptr(out), N.ptr(sc), st), "ab_gmm_ll_mod")
        return float(out.item())

    def pred_ll(self, Y_test, stream=None):
        """Log-likelihood of test points under the current weights, means and
        covariances: sum_n log sum_k pis[k] N(y_n | mu_k, cov_k) (inner_ll of
        experiments/hmvgmm/hmvgmm.py:143-178), on the device."""
        Y_test = np.ascontiguousarray(Y_test, np.float32)
        if Y_test.ndim != 2 or Y_test.shape[1] != self.d:
            raise ValueError("test points must be [n, %d]" % self.d)
        st = N.stream_ptr(stream)
        self._refresh_tables(st)
        sc, out = self._ll_buffers()
        Yd = torch.as_tensor(Y_test).to(self.Y.device)
        N.check(N.lib().ab_gmm_pred_ll(Y_test.shape[0], self.d, self.K, int(self.shared), N.ptr(Yd), N.ptr(self.pis),
                                       N.ptr(self.mu), N.ptr(self.Linv), N.ptr(self.hdet), N.ptr(out), N.ptr(sc),
                                       st), "ab_gmm_pred_ll")
        return float(out.item())

    # ---- one augur_step ----------------------------------------------------
    @traced("gmm.sweep")
    def sweep(self, n=1, stream=None):
        L = N.lib()
        st = N.stream_ptr(stream)
        d, K = self.d, self.K
        for _ in range(int(n)):
            it = self.iteration
            if self.shared:
                if self.move == "conj":
                    N.check(L.ab_gmm_stats(self.N, d, K, N.ptr(self.Y), N.ptr(self.z), None, N.ptr(self.cnt),
                                           N.ptr(self.sum), None, N.ptr(self.scratch), st), "stats")
                    N.check(L.ab_gmm_conj_mu(K, d, 1, N.ptr(self.mu0), N.ptr(self.cov0), N.ptr(self.cnt),
                                             N.ptr(self.sum), N.ptr(self.cov), N.ptr(self.mu), self.seed, it, 0,
                                             st), "conj_mu")
                elif self.move == "eslice":
                    N.check(L.ab_gmm_eslice(self.N, d, K, 1, N.ptr(self.Y), N.ptr(self.z), N.ptr(self.mu0),
                                            N.ptr(self.cov0), N.ptr(self.Linv), N.ptr(self.hdet), self.Kc,
                                            N.ptr(self.mu), self.seed, it, 0, N.ptr(self.shrinks), st), "eslice")
                else:
                    N.check(L.ab_gmm_mwg(self.N, d, K, 1, N.ptr(self.Y), N.ptr(self.z), N.ptr(self.mu0),
                                         N.ptr(self.prop_cov), N.ptr(self.Linv), N.ptr(self.hdet), self.Kc,
                                         self.Kc + 1, int(self.compat), N.ptr(self.mu), self.seed, it, 0,
                                         N.ptr(self.accepts), st), "mwg")
            else:
                N.check(L.ab_gmm_stats(self.N, d, K, N.ptr(self.Y), N.ptr(self.z), None, N.ptr(self.cnt),
                                       N.ptr(self.sum), None, N.ptr(self.scratch), st), "stats")
                # the Bartlett chi-square sums need only the counts: they are
                # drawn on a side stream beside the weights, the means and the
                # scatter pass (ab_gmm_conj_cov's draw, in two calls)
                main = stream if stream is not None else torch.cuda.current_stream(self.Y.device)
                if self._side is None:
                    self._side = torch.cuda.Stream(self.Y.device)
                fork = torch.cuda.Event()
                fork.record(main)
                self._side.wait_event(fork)
                N.check(L.ab_gmm_bartlett(K, d, self.df, N.ptr(self.cnt), N.ptr(self.chi), self.seed, it, 0,
                                          N.stream_ptr(self._side)), "bartlett")
                join = torch.cuda.Event()
                join.record(self._side)
                N.check(L.ab_gmm_conj_pis(K, N.ptr(self.alpha), N.ptr(self.cnt), N.ptr(self.pis), self.seed, it,
                                          0, st), "conj_pis")
                N.check(L.ab_gmm_conj_mu(K, d, 0, N.ptr(self.mu0), N.ptr(self.cov0), N.ptr(self.cnt),
                                         N.ptr(self.sum), N.ptr(self.cov), N.ptr(self.mu), self.seed, it, 0, st),
                        "conj_mu")
                N.check(L.ab_gmm_stats(self.N, d, K, N.ptr(self.Y), N.ptr(self.z), N.ptr(self.mu),
                                       N.ptr(self.cnt), None, N.ptr(self.obs), N.ptr(self.scratch), st), "stats")
                main.wait_event(join)
                N.check(L.ab_gmm_conj_cov_chi(K, d, self.df, N.ptr(self.scale0), N.ptr(self.cnt),
                                              N.ptr(self.obs), N.ptr(self.chi), N.ptr(self.cov), self.seed, it, 0,
                                              st), "conj_cov")
                N.check(L.ab_gmm_prep(K, d, N.ptr(self.cov), N.ptr(self.Linv), N.ptr(self.hdet), st), "prep")
            N.check(L.ab_gmm_disc_z_screened(self.N, d, K, int(self.shared), N.ptr(self.Y), N.ptr(self.pis),
                                             N.ptr(self.mu), N.ptr(self.Linv), N.ptr(self.hdet), N.ptr(self.z),
                                             self.seed, it, 0, N.ptr(self.zscratch), st), "disc_z")
            self.iteration += 1

    def state(self):
        out = {"mu": self.mu.cpu().numpy(), "z": self.z.cpu().numpy(), "pis": self.pis.cpu().numpy()}
        if not self.shared:
            out["cov"] = self.cov.cpu().numpy()
        return out

    def set_state(self, mu=None, z=None, pis=None, cov=None):
        if mu is not None:
            self.mu.copy_(torch.as_tensor(np.asarray(mu, np.float64)))
        if z is not None:
            self.z.copy_(torch.as_tensor(np.asarray(z, np.int32)))
        if pis is not None:
            self.pis.copy_(torch.as_tensor(np.asarray(pis, np.float64)))
        if cov is not None and not self.shared:
            self.cov.copy_(torch.as_tensor(np.asarray(cov, np.float64)))
