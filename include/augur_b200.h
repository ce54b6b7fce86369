/*
 * augur_b200.h - C ABI of the B200 (sm_100a) backend for the MCMC samplers
 * that AugurV2 compiles.
 *
 * In the reference, the Python front end (pyaugur/pyaugur/augurlib.py:
 * 445-519) loads a per-model library generated by the Haskell compiler and
 * calls augur_iface_init / augur_step / augur_cpy / augur_set_pt /
 * augur_get_curr_ll through ctypes (compiler/augur/src/CudaC/CgStInit.hs:
 * 474-602, CgKern.hs:232-238).  Those functions run the kernels of
 * cbits/augur_mcmclib.h over generated log-density, gradient and Gibbs
 * functions.  This library replaces that generated code and the cbits
 * runtime with hand-written CUDA: each entry point below names the reference
 * function or generated function it stands in for.
 *
 * Conventions (all entry points):
 *  - plain C types only; arrays are DEVICE pointers owned by the caller;
 *  - every call is enqueued on the caller's CUDA stream (`stream`, a
 *    cudaStream_t passed as void*; NULL is the legacy default stream);
 *  - the return value is a status (AB_OK == 0); on failure
 *    ab_last_error() describes it.  Nothing calls exit();
 *  - random draws come from Philox4x32-10 substreams addressed by
 *    (draw, element, iteration, tag) under the 64-bit seed, so results are
 *    reproducible and independent of launch shapes.
 */
#ifndef AUGUR_B200_H
#define AUGUR_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ------------------------------------------------------------ */
enum {
  AB_OK = 0,
  AB_ERR_ARG = 1,      /* invalid argument (sizes, null pointers)          */
  AB_ERR_CUDA = 2,     /* a CUDA runtime call or launch failed              */
  AB_ERR_TIMEOUT = 3,  /* a bounded device-side wait gave up                */
  AB_ERR_NUMERIC = 4,  /* non-finite value detected where one is forbidden  */
  AB_ERR_STATE = 5     /* call not valid in the object's current state      */
};

/* Divergence bound of every HMC / NUTS sampler: a transition whose energy
 * error (H_end - H_start) exceeds it, or is not finite, is counted as
 * divergent (for NUTS, a leaf whose log density falls below the slice level
 * by more than it: the reference's deltaMax, cbits/augur_mcmclib.h:152).
 * Divergent transitions are rejected by the accept test in any case; the
 * count is a diagnostic. */
#define AB_DIVERGENCE_DH 1000.0

/* Message of the calling thread's last failed call ("" if none).
 * Replaces the reference's exit()-on-error (cbits/augur_util.c:30-36). */
const char* ab_last_error(void);
/* Library version string. */
const char* ab_version(void);

/* ======================================================================= *
 * LDA Gibbs (model compiler/augur/test/lda.rv, schedule
 *   ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z])
 * Layouts: w, z int32[T] (documents contiguous); doc_off int32[D+1];
 * theta f64[D][K]; phiT f64[V][Kp] word-major with Kp = ab_lda_phi_stride(K),
 * 16-byte aligned, padding columns zero; theta and phi hold probabilities
 * (nonnegative); cnt_dk int32[D][K]; cnt_kw int32[K][V].
 * ======================================================================= */

/* Row stride (in doubles) of phiT for K topics. */
int ab_lda_phi_stride(int K);

/* Count statistics of z: replaces the generated conj_stat_theta and
 * conj_stat_phi (CgConj.hs:171-177) with the reset of CgKern.hs:103-107.
 * Overwrites both tables. */
int ab_lda_count(int D, int K, int V, const int* doc_off, const int* w, const int* z,
                 int* cnt_dk, int* cnt_kw, void* stream);

/* theta[d] ~ Dirichlet(alpha + cnt_dk[d]) for every d: replaces the generated
 * conj_samp_theta (CgConj.hs:278-299) over augur_dirichlet_categorical_conj
 * (cbits/augur_dist.c:526-538).  Element (d,k) draws from substream
 * (d*K+k, iter, 2). */
int ab_lda_conj_theta(int D, int K, const double* alpha, const int* cnt_dk, double* theta,
                      uint64_t seed, uint32_t iter, void* stream);

/* phi[k] ~ Dirichlet(beta + cnt_kw[k]) stored as phiT: replaces conj_samp_phi.
 * Element (k,v) draws from substream (k*V+v, iter, 3).  clear_counts != 0
 * zeroes cnt_kw after reading it.  `scratch` is caller-allocated device
 * memory of ab_lda_phi_scratch_bytes(K, V) bytes (per-CTA partial sums of
 * the gamma draws, per-topic normalisers and completion tickets); calls
 * sharing one scratch buffer must not overlap. */
size_t ab_lda_phi_scratch_bytes(int K, int V);
int ab_lda_conj_phi(int K, int V, const double* beta, int* cnt_kw, double* phiT,
                    int clear_counts, uint64_t seed, uint32_t iter, void* scratch, void* stream);

/* Same draw as ab_lda_conj_phi for callers that cannot allocate device
 * memory (a host framework that owns all device memory through its own pool,
 * or a plugin that must not allocate while it runs).  This entry point has no
 * counterpart in the reference.  It calls no cudaMalloc / cudaFree: its
 * scratch is a 1 MiB array inside the library that every GPU loading the
 * library keeps until the process exits, so it accepts only K, V with
 * ab_lda_phi_scratch_bytes(K, V) <= 1 MiB (K = 50, V = 10,000 needs 17 KB)
 * and rejects larger sizes with AB_ERR_ARG.  The first call on a device looks
 * up the array's device address; make that first call before any stream
 * capture.  The address is cached per device for the life of the process: a
 * cudaDeviceReset (or any other teardown of the device's primary context)
 * leaves the cached address stale, so do not call this entry point again in
 * a process that has reset the device.  All calls share the array: calls
 * whose work overlaps on the GPU (other streams, other threads) race and must
 * be serialised by the caller. */
int ab_lda_conj_phi_noalloc(int K, int V, const double* beta, int* cnt_kw, double* phiT,
                            int clear_counts, uint64_t seed, uint32_t iter, void* stream);

/* z[t] ~ p(z | theta, phi) for every token: replaces the generated disc_z
 * (CgDisc.hs:122-156) over augur_unnorm_disc_samp (cbits/augur_dist.c:
 * 798-813); token t draws one uniform from substream (t, iter, 1).  If the
 * count tables are given, cnt_dk is overwritten with the counts of the new z
 * and the counts of the new z are ADDED to cnt_kw (pass it zeroed). */
int ab_lda_disc_z(int D, int K, int V, const int* doc_off, const int* w, const double* theta,
                  const double* phiT, int* z, int* cnt_dk, int* cnt_kw, uint64_t seed,
                  uint32_t iter, void* stream);

/* The same draw screened in binary32 (K <= 64): phi32 f32 [V][Kq],
 * Kq = ab_lda_phi32_stride(K), 16-byte aligned, must hold phiT's values
 * rounded to nearest binary32 with zero padding (the sweep runner's phi
 * normalisation writes it).  Products and running sums are binary32 with a
 * margin that bounds their rounding, so every draw the screen decides equals
 * the reference's; the rest (u within the margin of a boundary, about 1e-5 of
 * the tokens at K = 50, or a degenerate norm) run the reference's binary64
 * loop on theta and phiT.  Results equal ab_lda_disc_z's bit for bit. */
int ab_lda_phi32_stride(int K);
int ab_lda_disc_z_f32(int D, int K, int V, const int* doc_off, const int* w, const double* theta,
                      const double* phiT, const float* phi32, int* z, int* cnt_dk, int* cnt_kw, uint64_t seed,
                      uint32_t iter, void* stream);

/* Sweep runner: the whole augur_step of the LDA schedule (CgKern.hs:232-238)
 * as a captured CUDA graph of four kernels (z screened in binary32 for
 * K <= 64). */
typedef struct ab_lda_desc {
  int D, K, V;
  const int* doc_off;   /* [D+1] */
  const int* w;         /* [T]   */
  const double* alpha;  /* [K]   */
  const double* beta;   /* [V]   */
  int* z;               /* [T]   */
  double* theta;        /* [D][K] */
  double* phiT;         /* [V][Kp] */
  int* cnt_dk;          /* [D][K] */
  int* cnt_kw;          /* [K][V] */
  void* scratch;        /* ab_lda_scratch_bytes(K, V) bytes of device memory */
  uint64_t seed;
} ab_lda_desc;

typedef struct ab_lda ab_lda;
/* Scratch of the sweep runner: its counters, the phi draw's partial sums and
 * normalisers, and the binary32 screening copy of phi (K <= 64). */
size_t ab_lda_scratch_bytes(int K, int V);
/* Replaces augur_iface_init for the LDA model (CgStInit.hs:474-510); the
 * caller owns every buffer named by the descriptor. */
int ab_lda_create(const ab_lda_desc* desc, ab_lda** out);
/* Sets the iteration counter and rebuilds the counts from the current z. */
int ab_lda_init_state(ab_lda* h, uint32_t iter, void* stream);
/* n_sweeps augur_step calls; use_graph selects graph replay. */
int ab_lda_run(ab_lda* h, int n_sweeps, int use_graph, void* stream);
int ab_lda_destroy(ab_lda* h);

/* ======================================================================= *
 * Hierarchical logistic regression (compiler/augur/test/hlr.rv; and the
 * variant with an InvGamma variance prior and no bias).  Parameters of one
 * chain: f64 par[D+2] = [theta[0..D-1], b, v].  A block is a list of indices
 * into par in the schedule's order (HMC [v, b, theta] -> D+1, D, 0..D-1).
 * ======================================================================= */
enum { AB_F32 = 0, AB_BF16 = 1 };

typedef struct ab_hlr_model {
  int N, D, ldx;        /* rows, features, row stride of X (elements)         */
  int has_b;            /* model has the bias b ~ Normal(0, v)                */
  int vprior;           /* 0: v ~ Exponential(lam); 1: v ~ InvGamma(a0, s0)   */
  int compat;           /* 1: the reference's own density formulas (its Normal
                           log density -log(var) - t^2/2var and dNormal/dvar)  */
  int x_dtype;          /* AB_F32 or AB_BF16                                  */
  double lam, a0, s0;
  const void* X;        /* device [N][ldx] */
  const int* y;         /* device [N]: 0/1 (Bernoulli) or counts >= 0 (Poisson) */
  /* The data factor, with t = theta . x[n] + b (zero-initialised: the
   * logistic model above).  AB_LIK_POISSON: y[n] ~ Poisson(exp(t))
   * (augur_poisson_ll, cbits/augur_dist.c:124-130, adjoint through exp);
   * AB_LIK_NORMAL: yr[n] ~ Normal(t, obs_var) with a fixed variance
   * (augur_normal_ll, :372-381; compat selects the reference's -log(var)
   * normaliser).  The reference's modelling language states these as
   * `data y[n] ~ Poisson(exp(dotprod(theta, x[n]) + b))` and
   * `data y[n] ~ Normal(dotprod(theta, x[n]) + b, s2)`. */
  int lik;              /* AB_LIK_BERNOULLI (0), AB_LIK_POISSON, AB_LIK_NORMAL */
  double obs_var;       /* AB_LIK_NORMAL: observation variance > 0 */
  const float* yr;      /* AB_LIK_NORMAL: device [N] real labels */
} ab_hlr_model;
enum { AB_LIK_BERNOULLI = 0, AB_LIK_POISSON = 1, AB_LIK_NORMAL = 2 };

/* One schedule component: kind 0 = HMC [block] [simlen, eps]
 * (h_augur_mcmc_hmc, cbits/augur_mcmclib.h:389-424), 1 = NUTS [block] [eps]
 * (h_augur_mcmc_nuts, :693-776; max_depth bounds the doublings), 2 = MWG on
 * one scalar with a Normal(x, mwg_var) proposal (augur_mcmc_mwg, :178-193),
 * 3 = RSlice [block] [simlen, eps] (h_augur_mcmc_refl_slice, :498-543).
 * The block is idx[idx_off .. idx_off+P-1] of the index array. */
typedef struct ab_hlr_comp {
  int kind, P, idx_off, max_depth;
  double simlen, eps, mwg_var;
} ab_hlr_comp;

/* Block log full-conditional and its gradient for C parameter vectors:
 * replaces the generated ll_<blk> / grad_<blk> functions (CgLike.hs:139-147,
 * CgGrad.hs:345-376).  ll f64[C]; grad f64[C][P] (may be NULL).  The block
 * indices are given both on the device (read by the kernel) and on the host
 * (validated). */
int ab_hlr_ll_grad(const ab_hlr_model* model, const int* idx_dev, const int* idx_host, int P, int C,
                   const double* pars, double* ll, double* grad, void* stream);

/* n_iter augur_step calls of a schedule of components for C independent
 * chains (one thread block per chain, the whole iteration on chip).
 * pars f64[C][D+2] in/out; stats f64[C][n_comps][AB_HLR_STATS] accumulates
 * {accepts (moves for RSlice), NUTS depth, NUTS leaves or RSlice
 * reflections, stack overflows, divergent HMC / NUTS iterations}.  scratch:
 * ab_hlr_chain_scratch_bytes(C, D) bytes, needed when a NUTS component is
 * present.  Substreams: momentum (c*P+j, iter, 4|comp<<8), HMC jitter and
 * accept (c, iter, 5|comp<<8), NUTS (c, iter, 6|comp<<8), MWG (c, iter,
 * 11|comp<<8), RSlice slice level (c, iter, 14|comp<<8). */
#define AB_HLR_STATS 5
size_t ab_hlr_chain_scratch_bytes(int C, int D);
int ab_hlr_run_chains(const ab_hlr_model* model, const ab_hlr_comp* comps_host, const void* comps_dev,
                      int n_comps, const int* idx_dev, const int* idx_host, int C, double* pars,
                      int n_iter, uint32_t iter0, uint64_t seed, double* stats, void* scratch,
                      void* stream);

/* ======================================================================= *
 * Gaussian mixtures (compiler/augur/test/mvgmm.rv: shared covariance, fixed
 * weights; hmvgmm.rv: weights ~ Dirichlet(alpha), cov[k] ~ InvWishart).
 * Layouts: Y f32 [N][d]; z int32 [N]; pis f64 [K]; mu f64 [K][d];
 * cov f64 [Kc][d][d] (Kc = 1 when shared); tables Linv f64 [slots][d][d] and
 * hdet f64 [slots].  Binary64 throughout; d <= 64, K <= 64.
 * ======================================================================= */

/* Per-covariance tables of augur_mvnormal_ll (cbits/augur_dist.c:548-568):
 * Linv = inverse of the lower Cholesky factor, hdet = log(det)/2, for Kc
 * covariances. */
size_t ab_gmm_table_doubles(int Kc, int d);
int ab_gmm_prep(int Kc, int d, const double* cov, double* Linv, double* hdet, void* stream);

/* z[n] ~ p(z | pis, mu, cov): replaces the generated disc_z with pmf_k =
 * pis[k] * augur_mvnormal_pdf(y_n, mu[k], cov[k]) and augur_unnorm_disc_samp
 * (CgDisc.hs:122-156); point n draws one uniform from (n, iter, 1|comp<<8). */
int ab_gmm_disc_z(int N, int d, int K, int shared_cov, const float* Y, const double* pis, const double* mu,
                  const double* Linv, const double* hdet, int* z, uint64_t seed, uint32_t iter, uint32_t comp,
                  void* stream);

/* The same draw decided for most points in binary32: log p_k per point and
 * component with a rigorous bound on its error (the binary32 rounding of
 * Linv, mu and y - mu, of every product and sum, and the reference's own
 * binary64 roundings), the running sums of p_k / p_max, and the reference's
 * draw wherever the uniform lies outside their uncertainty band; the other
 * points (a few in 10^4), and every point of a call with extreme
 * log-densities, run the reference's binary64 loop.  Equal to
 * ab_gmm_disc_z bit for bit.  scratch: ab_gmm_z_scratch_bytes(N, d, K)
 * bytes, 256-byte aligned (component tables and the queue of points the
 * screen leaves).  Shapes outside K <= 32, d <= 32 run ab_gmm_disc_z's
 * kernel. */
size_t ab_gmm_z_scratch_bytes(int N, int d, int K);
/* Byte offset in that scratch of an int: how many points of the last call
 * took the binary64 path (when the screen ran). */
size_t ab_gmm_z_queue_offset(int d, int K);
int ab_gmm_disc_z_screened(int N, int d, int K, int shared_cov, const float* Y, const double* pis,
                           const double* mu, const double* Linv, const double* hdet, int* z, uint64_t seed,
                           uint32_t iter, uint32_t comp, void* scratch, void* stream);

/* Conjugate statistics of z (CgConj.hs:186-246): counts cnt int32 [K] always;
 * sum f64 [K][d] of y if `sum` is non-NULL; obs f64 [K][d][d] =
 * sum (y - mu[z])(y - mu[z])^T if `obs` is non-NULL (needs mu).  scratch:
 * ab_gmm_stats_scratch_bytes(d, K) bytes (per-block partial tables). */
size_t ab_gmm_stats_scratch_bytes(int d, int K);
int ab_gmm_stats(int N, int d, int K, const float* Y, const int* z, const double* mu, int* cnt, double* sum,
                 double* obs, void* scratch, void* stream);

/* ConjGibbs [pis]: Dirichlet(alpha + cnt) (augur_dirichlet_categorical_conj,
 * cbits/augur_dist.c:526-538), element k from (k, iter, 7|comp<<8). */
int ab_gmm_conj_pis(int K, const double* alpha, const int* cnt, double* pis, uint64_t seed, uint32_t iter,
                    uint32_t comp, void* stream);

/* ConjGibbs [mu]: augur_mvnormal_mvnormal_conj (cbits/augur_dist.c:633-669)
 * per component with covariance cov[shared ? 0 : k]; (k, iter, 8|comp<<8). */
int ab_gmm_conj_mu(int K, int d, int shared_cov, const double* mu0, const double* cov0, const int* cnt,
                   const double* sum, const double* cov, double* mu, uint64_t seed, uint32_t iter, uint32_t comp,
                   void* stream);

/* ConjGibbs [cov]: augur_invwishart_mvnormal_conj (cbits/augur_dist.c:751-757,
 * InvWishart(cnt + df, obs + scale0) by Bartlett); (k, iter, 9|comp<<8).
 * cov is output only: its diagonal holds the Bartlett chi-square sums
 * between the two kernels of the call. */
int ab_gmm_conj_cov(int K, int d, int df, const double* scale0, const int* cnt, const double* obs, double* cov,
                    uint64_t seed, uint32_t iter, uint32_t comp, void* stream);

/* The same draw in two calls, so that the first can run beside the steps
 * that still read cov (the conjugate mean draw and the scatter pass):
 * ab_gmm_bartlett writes the Bartlett chi-square sums (bartlett_decomp's
 * diagonal before its square root, cbits/augur_dist.c:722-738) into chi
 * double[K][d]; ab_gmm_conj_cov_chi then makes the draw from them.  Together
 * they give ab_gmm_conj_cov's result bit for bit. */
int ab_gmm_bartlett(int K, int d, int df, const int* cnt, double* chi, uint64_t seed, uint32_t iter,
                    uint32_t comp, void* stream);
int ab_gmm_conj_cov_chi(int K, int d, int df, const double* scale0, const int* cnt, const double* obs,
                        const double* chi, double* cov, uint64_t seed, uint32_t iter, uint32_t comp, void* stream);

/* ESlice [mu]: augur_mcmc_eslice (cbits/augur_mcmclib.h:439-485) for every
 * component (one thread block each) over the full conditional of mu[k]
 * (prior table in slot prior_slot); (k, iter, 10|comp<<8).  shrinks int32[K]. */
int ab_gmm_eslice(int N, int d, int K, int shared_cov, const float* Y, const int* z, const double* mu0,
                  const double* cov0, const double* Linv, const double* hdet, int prior_slot, double* mu,
                  uint64_t seed, uint32_t iter, uint32_t comp, int* shrinks, void* stream);

/* MWG [mu] ~ MvNormal(mu[k], covp) (augur_mcmc_mwg, cbits/augur_mcmclib.h:
 * 178-193, generated prop_/swap_ of CgUserProp.hs:131-210); compat uses the
 * generated log-correction.  (k, iter, 11|comp<<8).  accepts int32[K] += . */
int ab_gmm_mwg(int N, int d, int K, int shared_cov, const float* Y, const int* z, const double* mu0,
               const double* covp, const double* Linv, const double* hdet, int prior_slot, int prop_slot,
               int compat, double* mu, uint64_t seed, uint32_t iter, uint32_t comp, int* accepts, void* stream);

/* ======================================================================= *
 * Whole-model log density (augur_get_curr_ll), held-out predictive
 * log-likelihoods, and dethlr's deterministic variable.
 * Each reduction writes one double to `out` (device memory) and needs
 * `scratch` of ab_ll_scratch_bytes() bytes of device memory, zero before the
 * first call (it returns to zero after each call); calls sharing a scratch
 * must not overlap.
 * ======================================================================= */
size_t ab_ll_scratch_bytes(void);

/* ll_mod of lda.rv: replaces the generated ll_mod behind augur_get_curr_ll
 * (CgStInit.hs:597-602): sum of augur_dirichlet_ll (no normalising constant,
 * cbits/augur_dist.c:488-496) over the theta rows (alpha) and phi rows
 * (beta), and augur_categorical_ll (:96-102) of every z and w. */
int ab_lda_ll_mod(int D, int K, int V, const int* doc_off, const int* w, const int* z, const double* alpha,
                  const double* beta, const double* theta, const double* phiT, double* out, void* scratch,
                  void* stream);

/* Predictive log-likelihood of held-out tokens (doc_off, w) for one theta
 * sample: sum over tokens of logsumexp_k(log theta[d][k] + log phi[k][w])
 * (experiments/lda/lda.py:149-173, the inner sum). */
int ab_lda_pred_ll(int D, int K, int V, const int* doc_off, const int* w, const double* theta,
                   const double* phiT, double* out, void* scratch, void* stream);

/* ll_mod of hmvgmm.rv (shared_cov = 0) or mvgmm.rv (shared_cov = 1), from the
 * component tables of ab_gmm_prep (Linv, hdet: [Kc] slots), the table of the
 * mean prior's covariance (Linv0, hdet0 [1]) and, for hmvgmm, the Dirichlet
 * alpha, the inverse-Wishart df and scale0 with its hdet_s0 [1] =
 * log(det scale0)/2 (ab_gmm_prep of scale0); all pointers are device memory:
 * augur_dirichlet_ll, augur_mvnormal_ll (:548-568), augur_invwishart_ll
 * (:679-711, with augur_multi_lgamma's log(3.1415)), augur_categorical_ll. */
int ab_gmm_ll_mod(int N, int d, int K, int shared_cov, const float* Y, const int* z, const double* pis,
                  const double* mu, const double* Linv, const double* hdet, const double* mu0,
                  const double* Linv0, const double* hdet0, const double* alpha, int df, const double* scale0,
                  const double* hdet_s0, double* out, void* scratch, void* stream);

/* Predictive log-likelihood of points Y [N][d] for one (pis, mu, cov) sample:
 * sum_n logsumexp_k(log N(y_n | mu_k, cov_k) + log pis[k])
 * (experiments/hmvgmm/hmvgmm.py:143-178, inner_ll). */
int ab_gmm_pred_ll(int N, int d, int K, int shared_cov, const float* Y, const double* pis, const double* mu,
                   const double* Linv, const double* hdet, double* out, void* scratch, void* stream);

/* dethlr.rv's deterministic bias[n] = sigmoid(dotprod(theta, x[n]) + b) for
 * C parameter vectors pars f64 [C][D+2]: out f64 [C][N] (replaces the
 * generated deterministic-variable code, CgDet.hs, with augur_dotprod and
 * augur_expit, cbits/augur_math.c:52-54,119-142). */
int ab_hlr_det(const ab_hlr_model* model, int C, const double* pars, double* out, void* stream);

/* ======================================================================= *
 * Batched HLR on the tensor cores: C chains against one data set.
 * The reference evaluates one chain's block log density and gradient with
 * its generated ll_/grad_ functions (compiler/augur/src/Comm/CgLike.hs:
 * 139-147, CgGrad.hs:345-376) over augur_bernoulli_ll / augur_dotprod
 * (cbits/augur_dist.c:59-71, cbits/augur_math.c:52-59,119-163); these entry
 * points compute the same quantities for every chain in two bf16 tensor-core
 * passes over the data (FP32-exact products by three-way bf16 splitting).
 * The prior on each coefficient is Normal(0, prior_a) or Student-t with
 * prior_a degrees of freedom and scale prior_b (no reference counterpart:
 * the reference's modelling language has no Student-t).
 * ======================================================================= */
enum { AB_PRIOR_NORMAL = 0, AB_PRIOR_STUDENT_T = 1 };

typedef struct ab_hlrb_model {
  int N, D, ldx;        /* rows, features, row stride of X (multiple of 8)    */
  const void* X;        /* bf16 [N][ldx], device                              */
  const void* Xt;       /* bf16 [Np/64][D][64] from ab_hlrb_transpose, device */
  const int* y;         /* int32 [N] labels 0/1, device                       */
  int prior;            /* AB_PRIOR_NORMAL or AB_PRIOR_STUDENT_T              */
  double prior_a, prior_b;
} ab_hlrb_model;

/* Elements of the transposed copy Xt: D x Np (Np = N rounded up to 64),
 * stored in 64-row blocks [Np/64][D][64]. */
size_t ab_hlrb_xt_elems(int N, int D);
int ab_hlrb_transpose(int N, int D, const void* X, int ldx, void* Xt, void* stream);
/* Device workspace (256-byte aligned) for ab_hlrb_logp_grad with C chains. */
size_t ab_hlrb_workspace_bytes(int N, int D, int C);
/* logp[c] (FP64) and grad[c][0..D-1] (FP32, row stride ldg) at
 * theta[c][0..D-1] (FP32, row stride ldt), for c < C.  Either output may be
 * NULL (not both): a NULL logp skips the log-likelihood terms (a leapfrog
 * step needs only the gradient), a NULL grad skips the backward pass. */
int ab_hlrb_logp_grad(const ab_hlrb_model* m, int C, const float* theta, int ldt, double* logp, float* grad,
                      int ldg, void* work, int* err, void* stream);

/* Launch shape of the batched pass, the knobs of the autotuner
 * (augurv2_b200/autotune.py); no reference counterpart (the reference's
 * gradient is a thrust reduction with no tiling, compiler/augur/src/Low/
 * SplitBlk.hs:382-389).  A zero field takes the built-in choice:
 *   fwd_warps   epilogue warps of the forward GEMM: 4, 8 or 16 (default 8)
 *   bwd_bn      gradient columns per backward tile: 32, 64 or 128 (default
 *               the narrowest that covers D)
 *   bwd_splits  row splits of the backward GEMM, >= 1 (default SMs / tiles)
 *   fwd_bn      data rows per forward tile: 128 or 256 (default 256)
 * Results of different shapes agree to FP32 rounding (the backward partial
 * sums are grouped differently); each shape is deterministic. */
typedef struct ab_hlrb_config {
  int fwd_warps, bwd_bn, bwd_splits, fwd_bn;
} ab_hlrb_config;
size_t ab_hlrb_workspace_bytes_cfg(int N, int D, int C, const ab_hlrb_config* cfg);
int ab_hlrb_logp_grad_cfg(const ab_hlrb_model* m, int C, const float* theta, int ldt, double* logp, float* grad,
                          int ldg, const ab_hlrb_config* cfg, void* work, int* err, void* stream);

/* ======================================================================= *
 * Batched HMC driver (h_augur_mcmc_hmc / h_augur_mcmc_leapfrog,
 * cbits/augur_mcmclib.h:343-424, for C chains at once).  All pointers are
 * device memory with row stride D; the caller evaluates the gradient (exact
 * or surrogate) between the calls:
 *   begin; { gradient at theta; step } x (L-1); exact logp + gradient; final
 * ======================================================================= */
#define AB_HMCB_STATS 3
typedef struct ab_hmcb_state {
  int C, D;
  unsigned long long seed;
  long long* iter;      /* iteration counter, advanced by ab_hmcb_final       */
  const float* eps0;    /* base step size                                     */
  float jitter;         /* eps_c = eps0 * (1 + jitter * (2u - 1)), in [0, 1)  */
  float* theta;         /* [C][D] current position                            */
  float* p;             /* [C][D] momentum                                    */
  float* g_cur;         /* [C][D] gradient used at the current position       */
  double* logp_cur;     /* [C] exact log density at the current position      */
  float* theta0;        /* [C][D] trajectory start (restored on reject)       */
  float* g0;            /* [C][D]                                             */
  double* logp0;        /* [C]                                                */
  double* H0;           /* [C] starting energy                                */
  float* eps_c;         /* [C] this iteration's step size                     */
  double* stats;        /* [C][AB_HMCB_STATS] accepted count, summed
                           acceptance probability, divergent transitions     */
} ab_hmcb_state;

int ab_hmcb_begin(const ab_hmcb_state* s, void* stream);
int ab_hmcb_step(const ab_hmcb_state* s, const float* g, void* stream);
int ab_hmcb_final(const ab_hmcb_state* s, const float* g_new, const double* logp_new, void* stream);

/* ======================================================================= *
 * Batched NUTS (h_augur_mcmc_nuts / h_augur_nuts_build_tree,
 * cbits/augur_mcmclib.h:575-776, for C chains of P parameters).  The chains'
 * resumable tree walks live in one device buffer of ab_nutsb_state_bytes;
 * each round is ab_nutsb_advance (every chain walks to its next leaf and
 * leaves the leaf position in the thprop array) followed by the caller's
 * evaluation of logp [C] and grad [C][P] at thprop, passed to the next
 * advance.  Completed iterations append their draws to a per-chain history
 * of hist_cap rows.  info[c][AB_NUTSB_INFO] = draws, last tree depth, last
 * leaves, error flag, iteration, mean depth, divergent iterations.
 * ======================================================================= */
#define AB_NUTSB_INFO 7
size_t ab_nutsb_state_bytes(int C, int P, int hist_cap);
int ab_nutsb_init(void* state, int C, int P, int hist_cap, const float* theta, const float* grad, const double* logp,
                  uint32_t iter0, void* stream);
int ab_nutsb_thprop(void* state, int C, int P, int hist_cap, float** thprop, float** hist, int** hist_depth);
int ab_nutsb_advance(void* state, int C, int P, int hist_cap, int max_depth, double eps, uint64_t seed, uint32_t comp,
                     const double* logp_new, const float* g_new, void* stream);
/* The same with a choice of selection rule.  AB_NUTS_REFERENCE is the
 * reference's (what ab_nutsb_advance runs): an iteration's draw is the pick
 * of its last doubling only (f_cpy reset per doubling,
 * cbits/augur_mcmclib.h:744-774) and the doubling's acceptance bias is
 * augur_min on the truncated ratio n'/n, so a chain moves only when the
 * final doubling is accepted whole.  AB_NUTS_STANDARD is Hoffman & Gelman's
 * efficient NUTS (2014, Algorithm 3): the latest accepted pick of any
 * doubling is the draw, accepted with probability min(1, n'/n).  Same tree
 * walk, leaves and random streams; no reference counterpart for the
 * standard rule. */
enum { AB_NUTS_REFERENCE = 0, AB_NUTS_STANDARD = 1 };
int ab_nutsb_advance_variant(void* state, int C, int P, int hist_cap, int max_depth, double eps, uint64_t seed,
                             uint32_t comp, int variant, const double* logp_new, const float* g_new, void* stream);
int ab_nutsb_info(void* state, int C, int P, int hist_cap, double* info, void* stream);
/* End of warm-up: the recorded draws are forgotten (draw counts and depth
 * statistics restart at zero) while every chain keeps its state; the
 * reference keeps no draw history of its own (pyaugur's samplen collects
 * draws on the host, pyaugur/augurlib.py:195-222). */
int ab_nutsb_reset_history(void* state, int C, int P, int hist_cap, void* stream);

/* ======================================================================= *
 * Many instances in one launch per stage.  The reference runs one chain of
 * one model per loaded library (process-global MCMC state,
 * cbits/augur_mcmclib.h:44-45), so it has no counterpart for grouping; each
 * instance's arithmetic is that of the single-instance calls above.
 *
 * ab_hlrg: the batched HLR pass (log density and gradient, the contract of
 * ab_hlrb_logp_grad) for n instances, each with its own data set and C_i
 * chains, one launch per stage covering every active instance.  When every
 * instance has D <= 256 the pass is FUSED: one persistent tensor-core kernel
 * runs forward, residual and backward per 128-row tile with the residual
 * kept in shared memory (no N x C scratch in HBM), the work units (chain
 * tile x 8192-row segment) of all instances balanced over the SMs; an
 * instance's results depend only on its own data, so they are the same
 * alone or in any group.  Otherwise the group runs the two-GEMM pass of
 * ab_hlrb_logp_grad (built-in launch shape) over all instances' tiles, equal
 * to each instance's own ab_hlrb_logp_grad bit for bit.  ab_hlrg_fused tells
 * which.  The group owns the workspaces; bind each instance's theta
 * [C_i][ldt] f32 input and logp [C_i] f64 / grad [C_i][ldg] f32 outputs,
 * then ab_hlrg_set_active (active[i] != 0 takes part) before the first pass
 * and after any change.  The tables live in device memory, so a CUDA graph
 * captured around ab_hlrg_logp_grad follows later ab_hlrg_set_active calls.
 * D_i must be a multiple of 8; n <= 256.
 * ======================================================================= */
typedef struct ab_hlrg ab_hlrg;
int ab_hlrg_create(int n, const ab_hlrb_model* models, const int* C, ab_hlrg** out);
int ab_hlrg_bind(ab_hlrg* g, int i, const float* theta, int ldt, double* logp, float* grad, int ldg);
int ab_hlrg_set_active(ab_hlrg* g, const int* active, void* stream);
int ab_hlrg_logp_grad(ab_hlrg* g, int* err, void* stream);
int ab_hlrg_fused(const ab_hlrg* g);
int ab_hlrg_destroy(ab_hlrg* g);

/* ab_nutsg: n batched-NUTS samplers advanced by one launch per round (each
 * instance's chains walk to their next leaf exactly as
 * ab_nutsb_advance_variant does, h_augur_mcmc_nuts,
 * cbits/augur_mcmclib.h:575-776).  A round is ab_nutsg_advance followed by
 * the caller's evaluation at every active instance's thprop (ab_hlrg for
 * HLR), written to the instance's logp_new / g_new.  ab_nutsg_min_draws
 * writes, for every instance (active or not), out[2i] = the smallest draw
 * count over its chains and out[2i+1] = 1 if any chain reported an error
 * (device int [2n]). */
typedef struct ab_nutsg_inst {
  void* state;              /* ab_nutsb_state_bytes buffer after ab_nutsb_init */
  int C, P, hist_cap, max_depth, variant;
  double eps;
  uint64_t seed;
  uint32_t comp;
  const double* logp_new;   /* [C] at thprop, from the caller's evaluation */
  const float* g_new;       /* [C][P] */
} ab_nutsg_inst;
typedef struct ab_nutsg ab_nutsg;
int ab_nutsg_create(int n, const ab_nutsg_inst* insts, ab_nutsg** out);
int ab_nutsg_set_active(ab_nutsg* g, const int* active, void* stream);
int ab_nutsg_advance(ab_nutsg* g, void* stream);
int ab_nutsg_min_draws(ab_nutsg* g, int* out, void* stream);
int ab_nutsg_destroy(ab_nutsg* g);

/* ======================================================================= *
 * Gradient-surrogate MLP (no counterpart in the reference): d_in -> h1 ->
 * h2 -> d_out, GELU hidden layers, flat FP32 master parameters w with a bf16
 * copy wb of the same layout [W1, b1, W2, b2, W3, b3]; forward passes use
 * the bf16 weights with FP32 accumulation.
 * ======================================================================= */
typedef struct ab_mlp_desc {
  int d_in, h1, h2, d_out;
  float* w;             /* FP32 master parameters, device                     */
  void* wb;             /* bf16 copy, device                                  */
} ab_mlp_desc;

size_t ab_mlp_param_count(int d_in, int h1, int h2, int d_out);
/* activation buffer (P1, A1, P2, A2) for a batch of B rows, in floats */
size_t ab_mlp_act_floats(int B, int h1, int h2);
size_t ab_mlp_backward_scratch_floats(int B, int h1, int h2);
int ab_mlp_forward(const ab_mlp_desc* d, int B, const float* x, int ldx, float* y, int ldy, float* act, void* stream);
/* dy = 2 (y - target) / (B D) (row stride D); row_sq[b] = squared error of row b */
int ab_mlp_mse(int B, int D, const float* y, int ldy, const float* target, int ldt, float* dy, double* row_sq,
               void* stream);
/* grad (flat, parameter layout) of the loss whose output gradient is dy */
int ab_mlp_backward(const ab_mlp_desc* d, int B, const float* x, int ldx, const float* dy, const float* act,
                    float* grad, float* scratch, void* stream);
int ab_mlp_adam(const ab_mlp_desc* d, const float* grad, float* m, float* v, int step, float lr, float b1, float b2,
                float eps, void* stream);
int ab_mlp_sync_bf16(const ab_mlp_desc* d, void* stream);
/* The surrogate in one launch: g = a + h (theta - mu) + o * MLP((theta - mu) * inv_s),
 * per coordinate, for C rows (d_in == d_out == D). */
int ab_sur_predict(const ab_mlp_desc* d, int C, const float* theta, int ldt, const float* mu, const float* inv_s,
                   const float* a, const float* h, const float* o, float* g, int ldg, void* stream);
/* Surrogate input/output maps around the network, per coordinate d:
 *   z = (theta - mu) * inv_s;   g = a + h (theta - mu) + o * out          */
int ab_sur_pre(int C, int D, const float* theta, const float* mu, const float* inv_s, float* z, void* stream);
int ab_sur_post(int C, int D, const float* theta, const float* out, const float* mu, const float* a, const float* h,
                const float* o, float* g, void* stream);

/* ======================================================================= *
 * Tensor-core building block (no counterpart in the reference, whose kernels
 * are scalar FP64): C[M][N] (f32, ldc) = A[M][K] * B[N][K]^T with A, B
 * row-major bf16, through tcgen05 MMAs fed by TMA.  splits > 1 splits K and
 * accumulates atomically.  *err (device int, may be NULL) receives
 * AB_ERR_TIMEOUT if a bounded wait inside the kernel expired.  Used by the
 * batched HLR data passes and the gradient surrogate, and exported for
 * checking the core on its own.
 * ======================================================================= */
int ab_tc_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                    int splits, int* err, void* stream);

/* Self-test of the kernels' bounded waits: one thread waits, through the
 * routine every tensor-core pipeline wait uses, on an mbarrier that nothing
 * completes, for at most limit_cycles SM cycles (at most the kernels' own
 * limit, about 2 s), then writes AB_ERR_TIMEOUT to *status and the cycles
 * it waited to *cycles (device pointers).  The context stays usable. */
int ab_tc_wait_probe(long long limit_cycles, int* status, long long* cycles, void* stream);

/* ======================================================================= *
 * Scalar conjugate Gibbs updates: the one-parameter conjugate pairs of the
 * reference library (cbits/augur_dist.c), which its compiler does not emit,
 * as one batched step over G groups.  Replaces, per group g,
 *   AB_CONJ_BETA_BERNOULLI     augur_beta_bernoulli_conj  (augur_dist.c:185-189)
 *                              p ~ Beta(h0 + sum, h1 + cnt - sum)
 *   AB_CONJ_BETA_GEOMETRIC     augur_beta_geometric_conj  (:191-195)
 *                              p ~ Beta(h0 + cnt, h1 + sum)
 *   AB_CONJ_GAMMA_POISSON      augur_gamma_poisson_conj   (:314-318)
 *                              l ~ Gamma(h0 + sum, rate h1 + cnt)
 *   AB_CONJ_GAMMA_EXPONENTIAL  augur_gamma_exponential_conj (:320-324)
 *                              l ~ Gamma(h0 + cnt, rate h1 + sum)
 *   AB_CONJ_GAMMA_GAMMASHAPE   augur_gamma_gammashape_conj (:326-330)
 *                              b ~ Gamma(h0 + sum aux, rate h1 + sum)
 *   AB_CONJ_GAMMA_INVGAMMA     augur_gamma_invgamma_conj  (:332-336)
 *                              b ~ Gamma(h0 + sum aux, rate h1 + sum 1/x)
 *   AB_CONJ_NORMAL_NORMALMEAN  augur_normal_normalmean_conj (:408-412)
 *                              m ~ Normal posterior of prior N(h0, h1) and
 *                              observations N(m, h2)
 * with cnt = off[g+1] - off[g] and sums over the group's observations
 * x[off[g] .. off[g+1]) (device, f64; aux = their known shapes for the
 * gammashape / invgamma kinds, else ignored).  h0, h1, h2 are device arrays
 * of G values (per_group = 1) or of one value (per_group = 0).  stat_sum /
 * stat_aux (optional, G doubles) receive the statistics (stat_aux = sum of
 * aux, or cnt).  Group g draws from Philox substream (g, iter, 15).
 * Posterior parameters that are not positive and finite give NaN.
 * ======================================================================= */
enum {
  AB_CONJ_BETA_BERNOULLI = 0,
  AB_CONJ_BETA_GEOMETRIC = 1,
  AB_CONJ_GAMMA_POISSON = 2,
  AB_CONJ_GAMMA_EXPONENTIAL = 3,
  AB_CONJ_GAMMA_GAMMASHAPE = 4,
  AB_CONJ_GAMMA_INVGAMMA = 5,
  AB_CONJ_NORMAL_NORMALMEAN = 6
};
int ab_conj_scalar(int kind, int G, const int* off, const double* x, const double* aux, const double* h0,
                   const double* h1, const double* h2, int per_group, double* stat_sum, double* stat_aux,
                   double* out, uint64_t seed, uint32_t iter, void* stream);

/* ======================================================================= *
 * Model handles: the generated module's entry points (augur_iface_init,
 * augur_step, augur_cpy, augur_set_pt, augur_get_curr_ll;
 * compiler/augur/src/CudaC/CgStInit.hs:474-602, called from
 * pyaugur/pyaugur/augurlib.py:445-519) as one opaque handle per model for
 * callers with host memory only.  ab_init_* copies the HOST arrays of the
 * descriptor into device memory the handle allocates and owns (as
 * augur_iface_init deep-copies its inputs, cbits/augur_rtmem.c:297-303);
 * ab_destroy frees it.  Handles share no state: several can live in one
 * process (the reference keeps one global chain, cbits/augur_mcmclib.h:
 * 44-45).  A failed call returns its status and its message is kept on the
 * handle (ab_model_last_error) as well as in ab_last_error().
 * ======================================================================= */
typedef struct ab_model ab_model;
enum { AB_MODEL_LDA = 1, AB_MODEL_HLR = 2, AB_MODEL_GMM = 3 };

/* lda.rv.  theta [D][K], phi [K][V], z [T] are the initial point (NULL:
 * uniform theta and phi, z = 0). */
typedef struct ab_lda_init {
  int D, K, V;
  const int* doc_off;     /* [D+1], doc_off[0] = 0 */
  const int* w;           /* [T = doc_off[D]], ids in [0, V) */
  const double* alpha;    /* [K] */
  const double* beta;     /* [V] */
  const double* theta;    /* [D][K] or NULL */
  const double* phi;      /* [K][V] or NULL */
  const int* z;           /* [T] or NULL */
  uint64_t seed;
  uint32_t iter0;
} ab_lda_init;
int ab_init_lda(const ab_lda_init* init, ab_model** out);

/* hlr.rv / dethlr.rv / the inverse-gamma variance variant: C chains of a
 * schedule of components (ab_hlr_comp, blocks indexing idx) on the per-chain
 * engine; X is stored in f32 on the device.  pars [C][D+2] = [theta, b, v]. */
typedef struct ab_hlr_init {
  int N, D, has_b, vprior, compat;
  double lam, a0, s0;
  const double* X;            /* [N][D] */
  const int* y;               /* [N], 0/1 */
  int C;
  const double* pars;         /* [C][D+2] initial point of every chain */
  int n_comps;
  const ab_hlr_comp* comps;   /* [n_comps] */
  const int* idx;             /* [n_idx] block indices */
  int n_idx;
  uint64_t seed;
  uint32_t iter0;
} ab_hlr_init;
int ab_init_hlr(const ab_hlr_init* init, ab_model** out);

/* mvgmm.rv (shared_cov = 1: fixed pis and covs [d][d]; move 0 = ConjGibbs,
 * 1 = ESlice, 2 = MWG with proposal covariance prop_cov) or hmvgmm.rv
 * (shared_cov = 0: pis, covs [K][d][d] initial, alpha, df, scale0; move 0).
 * Y is stored in f32 on the device. */
typedef struct ab_gmm_init {
  int N, d, K, shared_cov, move, compat;
  const double* Y;            /* [N][d] */
  const double* mu0;          /* [d] */
  const double* cov0;         /* [d][d] */
  const double* pis;          /* [K] */
  const double* covs;         /* [d][d] (mvgmm) or [K][d][d] (hmvgmm) */
  const double* alpha;        /* [K] (hmvgmm) */
  int df;                     /* (hmvgmm) */
  const double* scale0;       /* [d][d] (hmvgmm) */
  const double* prop_cov;     /* [d][d] (MWG) */
  const double* mu;           /* [K][d] initial */
  const int* z;               /* [N] initial */
  uint64_t seed;
  uint32_t iter0;
} ab_gmm_init;
int ab_init_gmm(const ab_gmm_init* init, ab_model** out);

int ab_model_kind(const ab_model* h);
const char* ab_model_last_error(const ab_model* h);
/* n_iters augur_step calls (CgKern.hs:232-238) on the caller's stream. */
int ab_step(ab_model* h, int n_iters, void* stream);
/* Iterations taken since ab_init_* (plus iter0): the Philox iteration index
 * of the next step. */
uint32_t ab_iteration(const ab_model* h);
/* The parameters in a host buffer of ab_state_bytes(h) bytes (augur_cpy /
 * augur_set_pt).  Layouts: LDA theta f64 [D][K], phi f64 [K][V], z int32 [T];
 * HLR pars f64 [C][D+2]; GMM pis f64 [K], mu f64 [K][d], cov f64 [K][d][d]
 * (hmvgmm only), z int32 [N].  Both calls finish before returning. */
size_t ab_state_bytes(const ab_model* h);
int ab_get_state(ab_model* h, void* host, size_t bytes, void* stream);
int ab_set_state(ab_model* h, const void* host, size_t bytes, void* stream);
/* The complete sampler state (parameters, statistics the next step reads,
 * iteration counter and seed) in a host buffer of ab_checkpoint_bytes(h)
 * bytes.  ab_restore into a handle made with the same ab_init_* descriptor
 * sizes continues the chain exactly as the uninterrupted run (every draw is
 * addressed by the iteration in the counter-based Philox stream). */
size_t ab_checkpoint_bytes(ab_model* h);
int ab_checkpoint(ab_model* h, void* host, size_t bytes, void* stream);
int ab_restore(ab_model* h, const void* host, size_t bytes, void* stream);
/* augur_get_curr_ll: the model log density of the current state, one value
 * per chain (ab_curr_ll_count: C for HLR, 1 otherwise), into host memory. */
int ab_curr_ll_count(const ab_model* h);
int ab_curr_ll(ab_model* h, double* host, int n, void* stream);
int ab_destroy(ab_model* h);

#ifdef __cplusplus
}
#endif
#endif /* AUGUR_B200_H */
