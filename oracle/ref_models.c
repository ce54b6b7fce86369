/*
 * ORACLE (test infrastructure only).
 *
 * Hand restatement of the per-model functions that the reference compiler
 * would generate for the models on the hot path, written against the
 * reference runtime (cbits/*.c, compiled in place from the reference
 * sources by oracle/Makefile; nothing of it is copied here).  Every
 * distribution, sampler and linear-algebra call below is the reference's own
 * function; only the loops that the compiler would emit are restated, with
 * the compiler file:line each follows.  The random numbers come from the GSL
 * shim (gsl_shim.c), positioned on the Philox substream of each element so
 * that the CUDA library and this code draw the same uniforms.
 *
 * Built only into oracle/_ref/libaugur_ref.so.  Used to pin the standalone
 * oracle (augur_oracle.c) and as the timed reference CPU baseline.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <augur_util.h>
#include <augur_rtval.h>
#include <augur_vecop.h>
#include <augur_matop.h>
#include <augur_math.h>
#include <augur_dist.h>
#include "gsl/gsl_rng.h"
#include "oracle_rng.h"

static gsl_rng* ref_rng(uint64_t seed) {
  static gsl_rng* r = NULL;
  orc_shim_set_seed(seed);
  if (r == NULL) r = gsl_rng_alloc(gsl_rng_default);
  return r;
}

static AugurVec_t dvec(double* p, int n) {
  AugurVec_t v;
  v.ty = AUGUR_DBL; v.stride = 0; v.elems = (uint_t)n; v.data = p;
  return v;
}

/* ------------------------------------------------------------------------
 * LDA  (model: compiler/augur/test/lda.rv; examples/lda.py:12-22)
 * --------------------------------------------------------------------- */

/* disc_z: CgDisc.hs:122-156.  For each token, for each topic k (the
 * marginalising variable), prob = 1; prob *= Categorical_pdf(k, theta[d]);
 * prob *= Categorical_pdf(w[d,n], phi[k]) (declaration order, CgDisc.hs:
 * 132-139); pmf[k] = prob; then z[d,n] = augur_unnorm_disc_samp(rng, pmf)
 * (augur_dist.c:798-813).  One uniform per token, substream (t, iter, Z). */
void ref_lda_disc_z(int D, int K, int V, const int* doc_off, const int* w,
                    const double* theta, const double* phi, int* z,
                    uint64_t seed, uint32_t iter) {
  gsl_rng* rng = ref_rng(seed);
  double* pmf = (double*)malloc(sizeof(double) * (size_t)K);
  AugurVec_t vpmf = dvec(pmf, K);
  for (int d = 0; d < D; ++d) {
    AugurVec_t th = dvec((double*)theta + (size_t)d * K, K);
    for (int t = doc_off[d]; t < doc_off[d + 1]; ++t) {
      for (int k = 0; k < K; ++k) {
        AugurVec_t ph = dvec((double*)phi + (size_t)k * V, V);
        double prob = 1.0;
        prob *= augur_categorical_pdf(k, &th);
        prob *= augur_categorical_pdf(w[t], &ph);
        pmf[k] = prob;
      }
      orc_shim_seek(rng, (uint32_t)t, iter, ORC_TAG_Z);
      z[t] = augur_unnorm_disc_samp(rng, &vpmf);
    }
  }
  free(pmf);
}

/* conj_stat_theta / conj_stat_phi: CgConj.hs:155-183 (Dirichlet-Categorical,
 * conjDirCat :171-177) after the reset of CgKern.hs:103-107: counts rebuilt
 * from zero.  phi's statistic indexes by z through the CatCond substitution
 * (CgConj.hs:106-109). */
void ref_lda_conj_stat(int D, int K, int V, const int* doc_off, const int* w,
                       const int* z, int* cnt_dk, int* cnt_kw) {
  memset(cnt_dk, 0, sizeof(int) * (size_t)D * K);
  memset(cnt_kw, 0, sizeof(int) * (size_t)K * V);
  for (int d = 0; d < D; ++d)
    for (int t = doc_off[d]; t < doc_off[d + 1]; ++t) {
      AUGUR_ATMINCI(cnt_dk + (size_t)d * K + z[t], 1);
      AUGUR_ATMINCI(cnt_kw + (size_t)z[t] * V + w[t], 1);
    }
}

/* conj_samp for a row-stacked Dirichlet block (CgConj.hs:278-299 ->
 * augur_dirichlet_categorical_conj, augur_dist.c:526-538): each element is
 * augur_gamma_sample(alpha_i + cnt_i, 1) (augur_dist.c:302-312), then the row
 * is normalised by the sequential sum.  Each element draws from its own
 * substream (row*cols + i, iter, tag). */
static void ref_dirichlet_rows(int rows, int cols, const double* alpha,
                               const int* cnt, double* out, uint64_t seed,
                               uint32_t iter, uint32_t tag) {
  gsl_rng* rng = ref_rng(seed);
  for (int r = 0; r < rows; ++r) {
    double* dst = out + (size_t)r * cols;
    double acc = 0.0;
    for (int i = 0; i < cols; ++i) {
      orc_shim_seek(rng, (uint32_t)((size_t)r * cols + i), iter, tag);
      double tmp = augur_gamma_sample(rng, alpha[i] + (double)cnt[(size_t)r * cols + i], 1.0);
      dst[i] = tmp;
      acc += tmp;
    }
    for (int i = 0; i < cols; ++i) dst[i] = dst[i] / acc;
  }
}

void ref_lda_conj_theta(int D, int K, const double* alpha, const int* cnt_dk,
                        double* theta, uint64_t seed, uint32_t iter) {
  ref_dirichlet_rows(D, K, alpha, cnt_dk, theta, seed, iter, ORC_TAG_THETA);
}

void ref_lda_conj_phi(int K, int V, const double* beta, const int* cnt_kw,
                      double* phi, uint64_t seed, uint32_t iter) {
  ref_dirichlet_rows(K, V, beta, cnt_kw, phi, seed, iter, ORC_TAG_PHI);
}

/* One augur_step for 'ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z]'
 * (CgKern.hs:144-178: per component reset -> stat -> samp, in schedule
 * order).  Both statistics are functions of z alone, so one count pass feeds
 * both conjugate draws. */
void ref_lda_sweeps(int D, int K, int V, const int* doc_off, const int* w,
                    const double* alpha, const double* beta, double* theta,
                    double* phi, int* z, int* cnt_dk, int* cnt_kw,
                    uint64_t seed, uint32_t iter0, int n_sweeps) {
  for (int s = 0; s < n_sweeps; ++s) {
    uint32_t it = iter0 + (uint32_t)s;
    ref_lda_conj_stat(D, K, V, doc_off, w, z, cnt_dk, cnt_kw);
    ref_lda_conj_theta(D, K, alpha, cnt_dk, theta, seed, it);
    ref_lda_conj_phi(K, V, beta, cnt_kw, phi, seed, it);
    ref_lda_disc_z(D, K, V, doc_off, w, theta, phi, z, seed, it);
  }
}

/* Direct access to single reference primitives, for the oracle pins. */
double ref_gamma_sample(double shape, double rate, uint64_t seed, uint32_t elem,
                        uint32_t iter, uint32_t tag) {
  gsl_rng* rng = ref_rng(seed);
  orc_shim_seek(rng, elem, iter, tag);
  return augur_gamma_sample(rng, shape, rate);
}

int ref_unnorm_disc_samp(const double* pmf, int K, uint64_t seed, uint32_t elem,
                         uint32_t iter, uint32_t tag) {
  gsl_rng* rng = ref_rng(seed);
  AugurVec_t v = dvec((double*)pmf, K);
  orc_shim_seek(rng, elem, iter, tag);
  return augur_unnorm_disc_samp(rng, &v);
}

/* ------------------------------------------------------------------------
 * HLR (compiler/augur/test/hlr.rv; InvGamma-variance variant without bias)
 * Restated generated ll_/grad_/prop_/swap_ functions over the reference's
 * distribution library, driven by the reference's own h_augur_mcmc_hmc,
 * h_augur_mcmc_nuts and augur_mcmc_mwg (cbits/augur_mcmclib.h).
 * Parameter vector par = [theta[0..D-1], b, v]; a block is an index list in
 * schedule order.  Only the reference's own (compat) densities exist here.
 * --------------------------------------------------------------------- */
#include <augur_mcmclib.h>
#include <augur_blkop.h>

typedef struct {
  int N, D, has_b, vprior;
  double lam, a0, s0;
  const double* X;
  const int* y;
  const int* idx;
  int P;
  double* gbuf;   /* adjoint block storage, block order */
} ref_hlr_t;

static ref_hlr_t g_hlr;

/* The likelihood of the data factor (the generated code differs only there):
 * 0 y[n] ~ Bernoulli(sigmoid(t)), 1 y[n] ~ Poisson(exp(t)), 2 yr[n] ~
 * Normal(t, obs_var) with a fixed variance; t = theta . x[n] + b.  Set before
 * each ref_hlr_* call (ref_glm_set). */
static int g_lik = 0;
static double g_obs_var = 1.0;
static const double* g_yr = 0;

void ref_glm_set(int lik, double obs_var, const double* yr) {
  g_lik = lik;
  g_obs_var = obs_var;
  g_yr = yr;
}

/* Data factor of row n at t, and the adjoint of t (the generated chain:
 * the distribution's dotarg1 times the link's derivative). */
static double ref_lik_ll(int n, double t) {
  if (g_lik == 1) return augur_poisson_ll(g_hlr.y[n], augur_exp(t));
  if (g_lik == 2) return augur_normal_ll(g_yr[n], t, g_obs_var);
  return augur_bernoulli_ll(g_hlr.y[n], augur_expit(t));
}
static double ref_lik_adj(int n, double t) {
  if (g_lik == 1) return augur_poisson_dotarg1(g_hlr.y[n], augur_exp(t)) * augur_exp(t);
  if (g_lik == 2) return augur_normal_dotarg1(g_yr[n], t, g_obs_var);
  return augur_bernoulli_dotarg1(g_hlr.y[n], augur_expit(t)) * augur_expit_grad_0(t);
}

static int in_blk(int lo, int hi) {
  for (int j = 0; j < g_hlr.P; ++j) if (g_hlr.idx[j] >= lo && g_hlr.idx[j] < hi) return 1;
  return 0;
}

static double hlr_vprior_ll(double v) {
  return g_hlr.vprior == 0 ? augur_exponential_ll(v, g_hlr.lam)
                           : augur_invgamma_ll(v, g_hlr.a0, g_hlr.s0);
}
static double hlr_vprior_dot(double v) {
  return g_hlr.vprior == 0 ? augur_exponential_dotpt(v, g_hlr.lam)
                           : augur_invgamma_dotpt(v, g_hlr.a0, g_hlr.s0);
}

/* ll_<blk>: CgLike.hs:139-147 (factors in model order, Pi -> MapRed). */
static double ref_hlr_ll_fn(AugurAux_t aux, AugurMod_t mod) {
  const int D = g_hlr.D;
  double* par = mod.par;
  double b = g_hlr.has_b ? par[D] : 0.0, v = par[D + 1];
  int in_th = in_blk(0, D), in_b = g_hlr.has_b && in_blk(D, D + 1), in_v = in_blk(D + 1, D + 2);
  AugurVec_t th = dvec(par, D);
  double ll = 0.0;
  if (in_v) ll += hlr_vprior_ll(v);
  if (g_hlr.has_b && (in_b || in_v)) ll += augur_normal_ll(b, 0.0, v);
  if (in_th || in_v) {
    double s = 0.0;
    for (int k = 0; k < D; ++k) s += augur_normal_ll(par[k], 0.0, v);
    ll += s;
  }
  if (in_th || in_b) {
    double s = 0.0;
    for (int n = 0; n < g_hlr.N; ++n) {
      AugurVec_t xn = dvec((double*)g_hlr.X + (size_t)n * D, D);
      double t = augur_dotprod(&th, &xn) + b;
      s += ref_lik_ll(n, t);
    }
    ll += s;
  }
  return ll;
}

/* grad_<blk>: CgGrad.hs:165-376; accumulates onto the zeroed adjoint block. */
static void ref_hlr_grad_fn(AugurAux_t aux, AugurMod_t mod) {
  const int D = g_hlr.D;
  double* par = mod.par;
  double b = g_hlr.has_b ? par[D] : 0.0, v = par[D + 1];
  int in_th = in_blk(0, D), in_b = g_hlr.has_b && in_blk(D, D + 1), in_v = in_blk(D + 1, D + 2);
  double* full = (double*)calloc((size_t)D + 2, sizeof(double));
  AugurVec_t th = dvec(par, D);
  double* dst = (double*)malloc(sizeof(double) * (size_t)D);
  AugurVec_t vdst = dvec(dst, D);
  if (in_v) full[D + 1] += hlr_vprior_dot(v);
  if (g_hlr.has_b && (in_b || in_v)) {
    if (in_b) full[D] += augur_normal_dotpt(b, 0.0, v);
    if (in_v) full[D + 1] += augur_normal_dotarg2(b, 0.0, v);
  }
  if (in_th || in_v) {
    for (int k = 0; k < D; ++k) {
      if (in_th) full[k] += augur_normal_dotpt(par[k], 0.0, v);
      if (in_v) full[D + 1] += augur_normal_dotarg2(par[k], 0.0, v);
    }
  }
  if (in_th || in_b) {
    for (int n = 0; n < g_hlr.N; ++n) {
      AugurVec_t xn = dvec((double*)g_hlr.X + (size_t)n * D, D);
      double t2 = augur_dotprod(&th, &xn) + b;
      double adj2 = ref_lik_adj(n, t2);
      if (in_b) full[D] += adj2 * 1;
      if (in_th) {
        augur_dotprod_grad_0(&vdst, adj2 * 1, &th, &xn);
        for (int k = 0; k < D; ++k) full[k] += dst[k];
      }
    }
  }
  for (int j = 0; j < g_hlr.P; ++j) g_hlr.gbuf[j] += full[g_hlr.idx[j]];
  free(full);
  free(dst);
}

/* A block over the entries idx of `base` (one AUGUR_DBL component per index,
 * which is how a block of scalars is grouped; the data layout is what the
 * block operations see). */
typedef struct { AugurBlk_t blk; AugurTyp_t* typs; void** ptrs; } ref_blk;

static ref_blk mk_blk_idx(double* base, const int* idx, int P) {
  ref_blk r;
  r.typs = (AugurTyp_t*)malloc(sizeof(AugurTyp_t) * P);
  r.ptrs = (void**)malloc(sizeof(void*) * P);
  for (int j = 0; j < P; ++j) { r.typs[j] = AUGUR_DBL; r.ptrs[j] = base + idx[j]; }
  h_augur_blk_mk_group(&r.blk, P, r.typs, r.ptrs);
  return r;
}

static ref_blk mk_blk_dense(double* base, int P) {
  ref_blk r;
  r.typs = (AugurTyp_t*)malloc(sizeof(AugurTyp_t) * P);
  r.ptrs = (void**)malloc(sizeof(void*) * P);
  for (int j = 0; j < P; ++j) { r.typs[j] = AUGUR_DBL; r.ptrs[j] = base + j; }
  h_augur_blk_mk_group(&r.blk, P, r.typs, r.ptrs);
  return r;
}

static void free_blk(ref_blk* r) {
  free(r->blk.typs); free(r->blk.blks); free(r->typs); free(r->ptrs);
}

static gsl_rng* g_aux_rng = NULL;

static void ref_hlr_setup(int N, int D, int has_b, int vprior, double lam, double a0, double s0,
                          const double* X, const int* y, const int* idx, int P, uint64_t seed) {
  orc_shim_set_seed(seed);
  if (g_aux_rng == NULL) {
    g_aux_rng = gsl_rng_alloc(gsl_rng_default);
    initMcmc();                 /* h_rng and MCMC defaults (deltaMax = 1000) */
  }
  g_hlr.N = N; g_hlr.D = D; g_hlr.has_b = has_b; g_hlr.vprior = vprior;
  g_hlr.lam = lam; g_hlr.a0 = a0; g_hlr.s0 = s0;
  g_hlr.X = X; g_hlr.y = y; g_hlr.idx = idx; g_hlr.P = P;
}

double ref_hlr_ll(int N, int D, int has_b, int vprior, double lam, double a0, double s0,
                  const double* X, const int* y, const double* par, const int* idx, int P) {
  ref_hlr_setup(N, D, has_b, vprior, lam, a0, s0, X, y, idx, P, 0);
  AugurAux_t aux; AugurMod_t mod;
  aux.rng = g_aux_rng; mod.par = (double*)par;
  return ref_hlr_ll_fn(aux, mod);
}

void ref_hlr_grad(int N, int D, int has_b, int vprior, double lam, double a0, double s0,
                  const double* X, const int* y, const double* par, const int* idx, int P, double* g) {
  ref_hlr_setup(N, D, has_b, vprior, lam, a0, s0, X, y, idx, P, 0);
  AugurAux_t aux; AugurMod_t mod;
  aux.rng = g_aux_rng; mod.par = (double*)par;
  memset(g, 0, sizeof(double) * P);
  g_hlr.gbuf = g;
  ref_hlr_grad_fn(aux, mod);
}

/* One HMC transition through the reference's h_augur_mcmc_hmc. */
int ref_hlr_hmc(int N, int D, int has_b, int vprior, double lam, double a0, double s0,
                const double* X, const int* y, double* par, const int* idx, int P, double simlen,
                double eps, uint64_t seed, uint32_t iter, uint32_t chain, uint32_t comp) {
  ref_hlr_setup(N, D, has_b, vprior, lam, a0, s0, X, y, idx, P, seed);
  const int NP = D + 2;
  double* prop = (double*)malloc(sizeof(double) * NP);
  double* mem = (double*)calloc((size_t)3 * P, sizeof(double));
  memcpy(prop, par, sizeof(double) * NP);
  g_hlr.gbuf = mem;
  ref_blk th0 = mk_blk_idx(par, idx, P), ths = mk_blk_idx(prop, idx, P);
  ref_blk gb = mk_blk_dense(mem, P), p0 = mk_blk_dense(mem + P, P), ps = mk_blk_dense(mem + 2 * P, P);
  AugurAux_t aux; AugurMod_t curr, pr;
  aux.rng = g_aux_rng; curr.par = par; pr.par = prop;
  orc_shim_seek_elementwise(g_aux_rng, chain * (uint32_t)P, iter, ORC_TAG_MOM | (comp << 8));
  orc_shim_seek(h_rng, chain, iter, ORC_TAG_HMC | (comp << 8));
  double before = par[idx[0]];
  MCMC.aux = aux; MCMC.curr = curr; MCMC.prop = pr;   /* as the generated init does */
  h_augur_mcmc_hmc(AUGUR_CPU, aux, curr, pr, &th0.blk, &ths.blk, &gb.blk, &p0.blk, &ps.blk, simlen,
                   eps, ref_hlr_grad_fn, ref_hlr_ll_fn);
  int moved = 0;
  for (int j = 0; j < P; ++j) if (par[idx[j]] != prop[idx[j]]) moved = 1;
  (void)before;
  free_blk(&th0); free_blk(&ths); free_blk(&gb); free_blk(&p0); free_blk(&ps);
  free(prop); free(mem);
  return !moved;   /* invariant curr == prop holds after the kernel; 1 = states agree */
}

/* One reflective-slice transition through the reference's
 * h_augur_mcmc_refl_slice (cbits/augur_mcmclib.h:498-543). */
void ref_hlr_rslice(int N, int D, int has_b, int vprior, double lam, double a0, double s0,
                    const double* X, const int* y, double* par, const int* idx, int P, double simlen,
                    double eps, uint64_t seed, uint32_t iter, uint32_t chain, uint32_t comp) {
  ref_hlr_setup(N, D, has_b, vprior, lam, a0, s0, X, y, idx, P, seed);
  const int NP = D + 2;
  double* prop = (double*)malloc(sizeof(double) * NP);
  double* mem = (double*)calloc((size_t)2 * P, sizeof(double));
  memcpy(prop, par, sizeof(double) * NP);
  g_hlr.gbuf = mem;
  ref_blk th0 = mk_blk_idx(par, idx, P), ths = mk_blk_idx(prop, idx, P);
  ref_blk gb = mk_blk_dense(mem, P), p0 = mk_blk_dense(mem + P, P);
  AugurAux_t aux; AugurMod_t curr, pr;
  aux.rng = g_aux_rng; curr.par = par; pr.par = prop;
  orc_shim_seek_elementwise(g_aux_rng, chain * (uint32_t)P, iter, ORC_TAG_MOM | (comp << 8));
  orc_shim_seek(h_rng, chain, iter, ORC_TAG_RSLICE | (comp << 8));
  MCMC.aux = aux; MCMC.curr = curr; MCMC.prop = pr;
  h_augur_mcmc_refl_slice(AUGUR_CPU, aux, curr, pr, &th0.blk, &ths.blk, &gb.blk, &p0.blk, simlen, eps,
                          ref_hlr_grad_fn, ref_hlr_ll_fn);
  free_blk(&th0); free_blk(&ths); free_blk(&gb); free_blk(&p0);
  free(prop); free(mem);
}

/* One NUTS transition through the reference's h_augur_mcmc_nuts.  The
 * reference prints its proposal stack at every inner node. */
void ref_hlr_nuts(int N, int D, int has_b, int vprior, double lam, double a0, double s0,
                  const double* X, const int* y, double* par, const int* idx, int P, double eps,
                  uint64_t seed, uint32_t iter, uint32_t chain, uint32_t comp) {
  ref_hlr_setup(N, D, has_b, vprior, lam, a0, s0, X, y, idx, P, seed);
  const int NP = D + 2;
  double* prop = (double*)malloc(sizeof(double) * NP);
  double* mem = (double*)calloc((size_t)7 * P, sizeof(double));
  memcpy(prop, par, sizeof(double) * NP);
  g_hlr.gbuf = mem;
  ref_blk th0 = mk_blk_idx(par, idx, P), thp = mk_blk_idx(prop, idx, P);
  ref_blk gb = mk_blk_dense(mem, P), work = mk_blk_dense(mem + P, P);
  ref_blk tm = mk_blk_dense(mem + 2 * P, P), mm = mk_blk_dense(mem + 3 * P, P);
  ref_blk tpl = mk_blk_dense(mem + 4 * P, P), mpl = mk_blk_dense(mem + 5 * P, P);
  ref_blk shape = mk_blk_dense(mem + 6 * P, P);
  AugurAux_t aux; AugurMod_t curr, pr;
  aux.rng = g_aux_rng; curr.par = par; pr.par = prop;
  orc_shim_seek_elementwise(g_aux_rng, chain * (uint32_t)P, iter, ORC_TAG_MOM | (comp << 8));
  orc_shim_seek(h_rng, chain, iter, ORC_TAG_NUTS | (comp << 8));
  MCMC.aux = aux; MCMC.curr = curr; MCMC.prop = pr;   /* as the generated init does */
  h_augur_mcmc_nuts(AUGUR_CPU, aux, curr, pr, &th0.blk, &thp.blk, &gb.blk, &work.blk, &tm.blk,
                    &mm.blk, &tpl.blk, &mpl.blk, &shape.blk, eps, ref_hlr_grad_fn, ref_hlr_ll_fn);
  free_blk(&th0); free_blk(&thp); free_blk(&gb); free_blk(&work); free_blk(&tm); free_blk(&mm);
  free_blk(&tpl); free_blk(&mpl); free_blk(&shape);
  free(prop); free(mem);
}

/* MWG on one scalar of par through augur_mcmc_mwg, with the generated
 * prop_/swap_ (CgUserProp.hs:131-186): x' ~ Normal(x, var), llCorrect =
 * ll(x; x, var) - ll(x'; x, var). */
static int g_mwg_which;
static double g_mwg_var, g_mwg_corr;

static void ref_mwg_prop(AugurAux_t aux, AugurMod_t curr, AugurMod_t prop) {
  double x = curr.par[g_mwg_which];
  double xp = augur_normal_sample(aux.rng, x, g_mwg_var);
  prop.par[g_mwg_which] = xp;
  g_mwg_corr = augur_normal_ll(x, x, g_mwg_var) - augur_normal_ll(xp, x, g_mwg_var);
}

static void ref_mwg_swap(AugurAux_t aux, AugurMod_t curr, AugurMod_t prop, int dir) {
  if (dir == 0) curr.par[g_mwg_which] = prop.par[g_mwg_which];
  else prop.par[g_mwg_which] = curr.par[g_mwg_which];
}

int ref_hlr_mwg(int N, int D, int has_b, int vprior, double lam, double a0, double s0,
                const double* X, const int* y, double* par, int which, double var, uint64_t seed,
                uint32_t iter, uint32_t chain, uint32_t comp) {
  static int one[1];
  one[0] = which;
  ref_hlr_setup(N, D, has_b, vprior, lam, a0, s0, X, y, one, 1, seed);
  const int NP = D + 2;
  double* prop = (double*)malloc(sizeof(double) * NP);
  memcpy(prop, par, sizeof(double) * NP);
  g_mwg_which = which; g_mwg_var = var;
  AugurAux_t aux; AugurMod_t curr, pr;
  aux.rng = g_aux_rng; curr.par = par; pr.par = prop;
  orc_shim_seek(g_aux_rng, chain, iter, ORC_TAG_MWG | (comp << 8));
  double before = par[which];
  MCMC.aux = aux; MCMC.curr = curr; MCMC.prop = pr;   /* as the generated init does */
  augur_mcmc_mwg(aux, curr, pr, &g_mwg_corr, ref_mwg_prop, ref_mwg_swap, ref_hlr_ll_fn);
  free(prop);
  return par[which] != before;
}

/* ------------------------------------------------------------------------
 * Gaussian mixtures (compiler/augur/test/mvgmm.rv, hmvgmm.rv): the generated
 * disc_z, conj_stat_/conj_samp_ for pis / mu / cov, eslice_mu and mwg_mu
 * restated over the reference's matrix and distribution library.
 * --------------------------------------------------------------------- */
typedef struct {
  int N, d, K, shared_cov;
  const double* Y;
  const double* mu0;
  const double* cov0;
  const double* alpha;
  int df;
  const double* scale0;
} ref_gmm_t;

static AugurMat_t dmat(double* p, int d) {
  AugurMat_t m;
  m.ty = AUGUR_DBL; m.row = (uint_t)d; m.col = (uint_t)d; m.data = p;
  return m;
}

void ref_gmm_disc_z(const ref_gmm_t* g, const double* pis, const double* mu, const double* cov, int* z,
                    uint64_t seed, uint32_t iter) {
  const int d = g->d, K = g->K;
  gsl_rng* rng = ref_rng(seed);
  double* pmf = (double*)malloc(sizeof(double) * K);
  double* Lb = (double*)malloc(sizeof(double) * d * d);
  double* wb = (double*)malloc(sizeof(double) * d);
  AugurVec_t vpmf = dvec(pmf, K), vpis = dvec((double*)pis, K), w = dvec(wb, d);
  AugurMat_t L = dmat(Lb, d);
  for (int n = 0; n < g->N; n++) {
    AugurVec_t y = dvec((double*)g->Y + (size_t)n * d, d);
    for (int k = 0; k < K; k++) {
      AugurVec_t mk = dvec((double*)mu + (size_t)k * d, d);
      AugurMat_t ck = dmat((double*)(g->shared_cov ? cov : cov + (size_t)k * d * d), d);
      double prob = 1.0;
      prob *= augur_categorical_pdf(k, &vpis);
      prob *= augur_mvnormal_pdf(&y, &mk, &ck, &L, &w);
      pmf[k] = prob;
    }
    orc_shim_seek(rng, (uint32_t)n, iter, ORC_TAG_Z);
    z[n] = augur_unnorm_disc_samp(rng, &vpmf);
  }
  free(pmf); free(Lb); free(wb);
}

/* conj_stat_* (CgConj.hs:186-246): counts, sum of y (augur_vec_atm_plus),
 * sum of (y - mu[z])(y - mu[z])^T (augur_vec_minus + augur_mat_atm_inc_vtmt). */
void ref_gmm_stats(const ref_gmm_t* g, const int* z, const double* mu, int* cnt, double* sum, double* obs) {
  const int d = g->d, K = g->K;
  memset(cnt, 0, sizeof(int) * K);
  if (sum) memset(sum, 0, sizeof(double) * K * d);
  if (obs) memset(obs, 0, sizeof(double) * K * d * d);
  double* db = (double*)malloc(sizeof(double) * d);
  AugurVec_t diff = dvec(db, d);
  for (int n = 0; n < g->N; n++) {
    const int k = z[n];
    AugurVec_t y = dvec((double*)g->Y + (size_t)n * d, d);
    AUGUR_ATMINCI(cnt + k, 1);
    if (sum) { AugurVec_t sk = dvec(sum + (size_t)k * d, d); augur_vec_atm_plus(&sk, &y); }
    if (obs) {
      AugurVec_t mk = dvec((double*)mu + (size_t)k * d, d);
      augur_vec_minus(&diff, &y, &mk);
      AugurMat_t ok = dmat(obs + (size_t)k * d * d, d);
      augur_mat_atm_inc_vtmt(&ok, &diff);
    }
  }
  free(db);
}

void ref_gmm_conj_pis(const ref_gmm_t* g, const int* cnt, double* pis, uint64_t seed, uint32_t iter) {
  ref_dirichlet_rows(1, g->K, g->alpha, cnt, pis, seed, iter, ORC_TAG_PI);
}

void ref_gmm_conj_mu(const ref_gmm_t* g, const int* cnt, double* sum, const double* cov, double* mu,
                     uint64_t seed, uint32_t iter) {
  const int d = g->d;
  gsl_rng* rng = ref_rng(seed);
  double* L0b = (double*)malloc(sizeof(double) * d * d);
  double* Lb = (double*)malloc(sizeof(double) * d * d);
  double* w0b = (double*)malloc(sizeof(double) * d);
  AugurMat_t L0 = dmat(L0b, d), L = dmat(Lb, d);
  AugurVec_t w0 = dvec(w0b, d);
  AugurVec_t mu0 = dvec((double*)g->mu0, d);
  AugurMat_t cov0 = dmat((double*)g->cov0, d);
  for (int k = 0; k < g->K; k++) {
    AugurVec_t res = dvec(mu + (size_t)k * d, d);
    AugurVec_t sk = dvec(sum + (size_t)k * d, d);
    AugurMat_t ck = dmat((double*)(g->shared_cov ? cov : cov + (size_t)k * d * d), d);
    orc_shim_seek(rng, (uint32_t)k, iter, ORC_TAG_MU);
    augur_mvnormal_mvnormal_conj(rng, &res, &mu0, &cov0, &sk, cnt[k], &ck, &L0, &w0, &L);
  }
  free(L0b); free(Lb); free(w0b);
}

void ref_gmm_conj_cov(const ref_gmm_t* g, const int* cnt, double* obs, double* cov, uint64_t seed,
                      uint32_t iter) {
  const int d = g->d;
  gsl_rng* rng = ref_rng(seed);
  double* Lb = (double*)malloc(sizeof(double) * d * d);
  double* Wb = (double*)malloc(sizeof(double) * d * d);
  double* db = (double*)malloc(sizeof(double) * d);
  AugurMat_t L = dmat(Lb, d), W = dmat(Wb, d), sc = dmat((double*)g->scale0, d);
  AugurVec_t diff = dvec(db, d);
  for (int k = 0; k < g->K; k++) {
    AugurMat_t res = dmat(cov + (size_t)k * d * d, d);
    AugurMat_t ok = dmat(obs + (size_t)k * d * d, d);
    orc_shim_seek(rng, (uint32_t)k, iter, ORC_TAG_COV);
    augur_invwishart_mvnormal_conj(rng, &res, g->df, &sc, &ok, cnt[k], &diff, &L, &W);
  }
  free(Lb); free(Wb); free(db);
}

void ref_gmm_sweep(const ref_gmm_t* g, double* pis, double* mu, double* cov, int* z, uint64_t seed,
                   uint32_t iter) {
  const int d = g->d, K = g->K;
  int* cnt = (int*)malloc(sizeof(int) * K);
  double* sum = (double*)malloc(sizeof(double) * K * d);
  double* obs = (double*)malloc(sizeof(double) * K * d * d);
  if (!g->shared_cov) {
    ref_gmm_stats(g, z, mu, cnt, NULL, NULL);
    ref_gmm_conj_pis(g, cnt, pis, seed, iter);
  }
  ref_gmm_stats(g, z, mu, cnt, sum, NULL);
  ref_gmm_conj_mu(g, cnt, sum, cov, mu, seed, iter);
  if (!g->shared_cov) {
    ref_gmm_stats(g, z, mu, cnt, NULL, obs);
    ref_gmm_conj_cov(g, cnt, obs, cov, seed, iter);
  }
  ref_gmm_disc_z(g, pis, mu, cov, z, seed, iter);
  free(cnt); free(sum); free(obs);
}

/* ll_mu(k) (llFnDeclOne): prior of mu[k] then the points of component k. */
static const ref_gmm_t* g_gmm;
static const double* g_gmm_cov;
static const int* g_gmm_z;
static int g_gmm_k;

static double ref_gmm_ll_mu_fn(AugurAux_t aux, AugurMod_t mod) {
  const int d = g_gmm->d, k = g_gmm_k;
  double* Lb = (double*)malloc(sizeof(double) * d * d);
  double* wb = (double*)malloc(sizeof(double) * d);
  AugurMat_t L = dmat(Lb, d);
  AugurVec_t w = dvec(wb, d);
  AugurVec_t muk = *AUGUR_VEC_GETV(mod.mu, k);
  AugurVec_t mu0 = dvec((double*)g_gmm->mu0, d);
  AugurMat_t cov0 = dmat((double*)g_gmm->cov0, d);
  AugurMat_t ck = dmat((double*)(g_gmm->shared_cov ? g_gmm_cov : g_gmm_cov + (size_t)k * d * d), d);
  double ll = 0.0;
  ll += augur_mvnormal_ll(&muk, &mu0, &cov0, &L, &w);
  double s = 0.0;
  for (int n = 0; n < g_gmm->N; n++)
    if (g_gmm_z[n] == k) {
      AugurVec_t y = dvec((double*)g_gmm->Y + (size_t)n * d, d);
      s += augur_mvnormal_ll(&y, &muk, &ck, &L, &w);
    }
  ll += s;
  free(Lb); free(wb);
  return ll;
}

/* eslice_mu (CgESlice.hs:93-144) over augur_mcmc_eslice. */
void ref_gmm_eslice(const ref_gmm_t* g, double* mu, const double* cov, const int* z, uint64_t seed,
                    uint32_t iter) {
  const int d = g->d, K = g->K;
  gsl_rng* rng = ref_rng(seed);
  double* prop = (double*)malloc(sizeof(double) * K * d);
  double* Lb = (double*)malloc(sizeof(double) * d * d);
  double* nub = (double*)malloc(sizeof(double) * d);
  AugurVec_t* rows_c = (AugurVec_t*)malloc(sizeof(AugurVec_t) * K);
  AugurVec_t* rows_p = (AugurVec_t*)malloc(sizeof(AugurVec_t) * K);
  memcpy(prop, mu, sizeof(double) * K * d);
  for (int k = 0; k < K; k++) { rows_c[k] = dvec(mu + (size_t)k * d, d); rows_p[k] = dvec(prop + (size_t)k * d, d); }
  AugurVec_t vc, vp;
  vc.ty = AUGUR_VEC; vc.stride = 0; vc.elems = K; vc.data = rows_c;
  vp.ty = AUGUR_VEC; vp.stride = 0; vp.elems = K; vp.data = rows_p;
  AugurVec_t mu0 = dvec((double*)g->mu0, d), nu = dvec(nub, d);
  AugurMat_t cov0 = dmat((double*)g->cov0, d), L = dmat(Lb, d);
  g_gmm = g; g_gmm_cov = cov; g_gmm_z = z;
  AugurAux_t aux; AugurMod_t curr, pr;
  aux.rng = rng; curr.mu = &vc; pr.mu = &vp;
  for (int k = 0; k < K; k++) {
    g_gmm_k = k;
    orc_shim_seek(rng, (uint32_t)k, iter, ORC_TAG_ESLICE);
    augur_mcmc_eslice(aux, curr, pr, rows_c + k, rows_p + k, &mu0, &cov0, &L, &nu, ref_gmm_ll_mu_fn);
  }
  free(prop); free(Lb); free(nub); free(rows_c); free(rows_p);
}

/* mwg_mu with the proposal MvNormal(mu[k], covp) (CgUserProp.hs:131-260). */
static const double* g_mwg_covp;
static double g_mwg_corr_mu;

static void ref_gmm_mwg_prop(AugurAux_t aux, AugurMod_t curr, AugurMod_t prop) {
  const int d = g_gmm->d, k = g_gmm_k;
  double* Lb = (double*)malloc(sizeof(double) * d * d);
  double* wb = (double*)malloc(sizeof(double) * d);
  AugurMat_t L = dmat(Lb, d), cp = dmat((double*)g_mwg_covp, d);
  AugurVec_t w = dvec(wb, d);
  AugurVec_t* ck = AUGUR_VEC_GETV(curr.mu, k);
  AugurVec_t* pk = AUGUR_VEC_GETV(prop.mu, k);
  augur_mvnormal_sample(aux.rng, pk, ck, &cp, &L, &w);
  g_mwg_corr_mu = augur_mvnormal_ll(ck, ck, &cp, &L, &w) - augur_mvnormal_ll(pk, ck, &cp, &L, &w);
  free(Lb); free(wb);
}

static void ref_gmm_mwg_swap(AugurAux_t aux, AugurMod_t curr, AugurMod_t prop, int dir) {
  const int d = g_gmm->d, k = g_gmm_k;
  AugurVec_t* ck = AUGUR_VEC_GETV(curr.mu, k);
  AugurVec_t* pk = AUGUR_VEC_GETV(prop.mu, k);
  if (dir == 0) memcpy(ck->data, pk->data, sizeof(double) * d);
  else memcpy(pk->data, ck->data, sizeof(double) * d);
}

void ref_gmm_mwg(const ref_gmm_t* g, double* mu, const double* cov, const int* z, const double* covp,
                 uint64_t seed, uint32_t iter) {
  const int d = g->d, K = g->K;
  gsl_rng* rng = ref_rng(seed);
  double* prop = (double*)malloc(sizeof(double) * K * d);
  AugurVec_t* rows_c = (AugurVec_t*)malloc(sizeof(AugurVec_t) * K);
  AugurVec_t* rows_p = (AugurVec_t*)malloc(sizeof(AugurVec_t) * K);
  memcpy(prop, mu, sizeof(double) * K * d);
  for (int k = 0; k < K; k++) { rows_c[k] = dvec(mu + (size_t)k * d, d); rows_p[k] = dvec(prop + (size_t)k * d, d); }
  AugurVec_t vc, vp;
  vc.ty = AUGUR_VEC; vc.stride = 0; vc.elems = K; vc.data = rows_c;
  vp.ty = AUGUR_VEC; vp.stride = 0; vp.elems = K; vp.data = rows_p;
  g_gmm = g; g_gmm_cov = cov; g_gmm_z = z; g_mwg_covp = covp;
  AugurAux_t aux; AugurMod_t curr, pr;
  aux.rng = rng; curr.mu = &vc; pr.mu = &vp;
  for (int k = 0; k < K; k++) {
    g_gmm_k = k;
    orc_shim_seek(rng, (uint32_t)k, iter, ORC_TAG_MWG);
    augur_mcmc_mwg(aux, curr, pr, &g_mwg_corr_mu, ref_gmm_mwg_prop, ref_gmm_mwg_swap, ref_gmm_ll_mu_fn);
  }
  free(prop); free(rows_c); free(rows_p);
}

/* Scalar conjugate updates over G groups through the reference's own
 * samplers (cbits/augur_dist.c:185-195, 314-336, 408-412); the statistics
 * loop is what a generated conj_stat would run (sequential over the
 * observations, CgConj.hs:100-164).  Kind numbering and substreams as
 * orc_conj_scalar. */
void ref_conj_scalar(int kind, int G, const int* off, const double* x, const double* aux,
                     const double* h0, const double* h1, const double* h2, int per_group,
                     double* stat_sum, double* stat_aux, double* out, uint64_t seed, uint32_t iter) {
  gsl_rng* rng = ref_rng(seed);
  for (int g = 0; g < G; ++g) {
    const int cnt = off[g + 1] - off[g];
    double sum = 0.0, asum = 0.0;
    int isum = 0;
    for (int n = off[g]; n < off[g + 1]; ++n) {
      if (kind <= 2) isum += (int)x[n];
      sum += kind == 5 ? 1.0 / x[n] : x[n];
      if (kind == 4 || kind == 5) asum += aux[n];
    }
    if (stat_sum) stat_sum[g] = kind <= 2 ? (double)isum : sum;
    if (stat_aux) stat_aux[g] = (kind == 4 || kind == 5) ? asum : (double)cnt;
    const int j = per_group ? g : 0;
    orc_shim_seek(rng, (uint32_t)g, iter, ORC_TAG_CONJ);
    switch (kind) {
      case 0: out[g] = augur_beta_bernoulli_conj(rng, isum, cnt, h0[j], h1[j]); break;
      case 1: out[g] = augur_beta_geometric_conj(rng, isum, cnt, h0[j], h1[j]); break;
      case 2: out[g] = augur_gamma_poisson_conj(rng, isum, cnt, h0[j], h1[j]); break;
      case 3: out[g] = augur_gamma_exponential_conj(rng, sum, cnt, h0[j], h1[j]); break;
      case 4: out[g] = augur_gamma_gammashape_conj(rng, sum, asum, h0[j], h1[j]); break;
      case 5: out[g] = augur_gamma_invgamma_conj(rng, sum, asum, h0[j], h1[j]); break;
      default: out[g] = augur_normal_normalmean_conj(rng, sum, cnt, h0[j], h1[j], h2[j]);
    }
  }
}

/* ------------------------------------------------------------------------
 * ll_mod (the function augur_get_curr_ll returns, CgStInit.hs:597-602):
 * the model's factors in model order, each the sum over its comprehension
 * (CgLike.hs:128-147), with the reference's _ll functions.
 * --------------------------------------------------------------------- */

double ref_lda_ll_mod(int D, int K, int V, const int* doc_off, const int* w, const int* z,
                      const double* alpha, const double* beta, const double* theta, const double* phi) {
  AugurVec_t va = dvec((double*)alpha, K), vb = dvec((double*)beta, V);
  double ll = 0.0, s = 0.0;
  for (int d = 0; d < D; d++) {
    AugurVec_t th = dvec((double*)theta + (size_t)d * K, K);
    s += augur_dirichlet_ll(&th, &va);
  }
  ll += s;
  s = 0.0;
  for (int k = 0; k < K; k++) {
    AugurVec_t ph = dvec((double*)phi + (size_t)k * V, V);
    s += augur_dirichlet_ll(&ph, &vb);
  }
  ll += s;
  s = 0.0;
  for (int d = 0; d < D; d++) {
    AugurVec_t th = dvec((double*)theta + (size_t)d * K, K);
    for (int t = doc_off[d]; t < doc_off[d + 1]; t++) s += augur_categorical_ll(z[t], &th);
  }
  ll += s;
  s = 0.0;
  for (int d = 0; d < D; d++)
    for (int t = doc_off[d]; t < doc_off[d + 1]; t++) {
      AugurVec_t ph = dvec((double*)phi + (size_t)z[t] * V, V);
      s += augur_categorical_ll(w[t], &ph);
    }
  ll += s;
  return ll;
}

double ref_gmm_ll_mod(const ref_gmm_t* g, const double* pis, const double* mu, const double* cov, const int* z) {
  const int d = g->d, K = g->K;
  double* Lb = (double*)malloc(sizeof(double) * d * d);
  double* Wb = (double*)malloc(sizeof(double) * d * d);
  double* wb = (double*)malloc(sizeof(double) * d);
  AugurMat_t L = dmat(Lb, d), W = dmat(Wb, d);
  AugurVec_t work = dvec(wb, d);
  AugurVec_t vpis = dvec((double*)pis, K), mu0 = dvec((double*)g->mu0, d);
  AugurMat_t cov0 = dmat((double*)g->cov0, d);
  double ll = 0.0, s = 0.0;
  if (!g->shared_cov) {
    AugurVec_t va = dvec((double*)g->alpha, K);
    ll += augur_dirichlet_ll(&vpis, &va);
  }
  for (int k = 0; k < K; k++) {
    AugurVec_t mk = dvec((double*)mu + (size_t)k * d, d);
    s += augur_mvnormal_ll(&mk, &mu0, &cov0, &L, &work);
  }
  ll += s;
  s = 0.0;
  if (!g->shared_cov) {
    AugurMat_t sc = dmat((double*)g->scale0, d);
    for (int k = 0; k < K; k++) {
      AugurMat_t ck = dmat((double*)cov + (size_t)k * d * d, d);
      s += augur_invwishart_ll(&ck, g->df, &sc, &L, &W);
    }
    ll += s;
    s = 0.0;
  }
  for (int n = 0; n < g->N; n++) s += augur_categorical_ll(z[n], &vpis);
  ll += s;
  s = 0.0;
  for (int n = 0; n < g->N; n++) {
    AugurVec_t y = dvec((double*)g->Y + (size_t)n * d, d);
    AugurVec_t mk = dvec((double*)mu + (size_t)z[n] * d, d);
    AugurMat_t ck = dmat((double*)(g->shared_cov ? cov : cov + (size_t)z[n] * d * d), d);
    s += augur_mvnormal_ll(&y, &mk, &ck, &L, &work);
  }
  ll += s;
  free(Lb); free(Wb); free(wb);
  return ll;
}
