/*
 * ORACLE (test infrastructure only).
 *
 * Standalone plain-C restatement of the reference algorithms on the hot path,
 * written from the reference's sources and its compiler's code-generation
 * rules (each function cites the file:line it follows), with no code of the
 * reference linked in.  It is the checker of the CUDA library: the parity
 * tests, __graft_entry__.smoke() and the CPU-baseline leg of bench.py call it
 * through ctypes (oracle/oracle.py).  Nothing in the product links or calls
 * it.  It is pinned against the reference's own runtime compiled from source
 * (oracle/_ref, ref_models.c) by bit-for-bit tests on the same substreams,
 * and against the golden vectors in tests/golden/ made from that build.
 *
 * Arithmetic is binary64 with no fused multiply-add (gcc -O2 -ffp-contract=off
 * on x86-64), which is how the reference's libcpu path computes.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_rng.h"

/* ------------------------------------------------------------------------
 * Scalar samplers
 * --------------------------------------------------------------------- */

/* Marsaglia & Tsang (2000) for shape >= 1, as cbits/augur_dist.c:287-300:
 * d = a - 1/3, c = 1/sqrt(9 d); loop { z ~ N(0,1); u ~ U; V = (1 + c z)^3;
 * accept if z > -1/c and log u < z^2/2 + d - d V + d log V } -> d V. */
static double orc_gamma_ge1(orc_stream* s, double alpha) {
  double d = alpha - 1.0 / 3.0;
  double c = 1.0 / sqrt(9 * d);
  for (;;) {
    double z = orc_normal(s);
    double u = orc_uniform(s);
    double V = (1.0 + c * z) * (1.0 + c * z) * (1.0 + c * z);
    if (z > -1.0 / c && log(u) < (0.5 * z * z) + d - (d * V) + (d * log(V))) return d * V;
  }
}

/* cbits/augur_dist.c:302-312: shape < 1 boosts through Gamma(shape + 1) and
 * u^(1/shape); the result is scaled by 1/rate. */
double orc_gamma(orc_stream* s, double shape, double rate) {
  double scale = 1.0 / rate;
  if (shape < 1.0) {
    double x = orc_gamma_ge1(s, shape + 1.0);
    double u = orc_uniform(s);
    return (x * pow(u, 1.0 / shape)) * scale;
  }
  return orc_gamma_ge1(s, shape) * scale;
}

/* cbits/augur_dist.c:798-813: one uniform, sequential normaliser, then the
 * first i whose running sum of pmf[j]/norm exceeds u (acc starts at
 * pmf[0]/norm; the test happens before adding pmf[i]/norm). */
int orc_unnorm_disc(orc_stream* s, const double* pmf, int K) {
  double u = orc_uniform(s);
  double norm = 0.0;
  for (int i = 0; i < K; ++i) norm += pmf[i];
  double acc = pmf[0] / norm;
  for (int i = 1; i < K; ++i) {
    if (u < acc) return i - 1;
    acc += pmf[i] / norm;
  }
  return K - 1;
}

double orc_gamma_sample(double shape, double rate, uint64_t seed, uint32_t elem,
                        uint32_t iter, uint32_t tag) {
  orc_stream s = orc_make(seed, elem, iter, tag);
  return orc_gamma(&s, shape, rate);
}

int orc_unnorm_disc_samp(const double* pmf, int K, uint64_t seed, uint32_t elem,
                         uint32_t iter, uint32_t tag) {
  orc_stream s = orc_make(seed, elem, iter, tag);
  return orc_unnorm_disc(&s, pmf, K);
}

/* Raw contract access for the known-answer tests. */
void orc_philox_block(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  orc_philox(ctr, k0, k1, out);
}

void orc_draws(uint64_t seed, uint32_t elem, uint32_t iter, uint32_t tag, int n,
               int normal, double* out) {
  orc_stream s = orc_make(seed, elem, iter, tag);
  for (int i = 0; i < n; ++i) out[i] = normal ? orc_normal(&s) : orc_uniform(&s);
}

/* ------------------------------------------------------------------------
 * LDA  (compiler/augur/test/lda.rv)
 * --------------------------------------------------------------------- */

/* disc_z, compiler/augur/src/Core/CgDisc.hs:122-156: pmf[k] =
 * (1 * theta[d][k]) * phi[k][w] in declaration order, then the unnormalised
 * discrete draw.  Substream (token, iter, Z). */
void orc_lda_disc_z(int D, int K, int V, const int* doc_off, const int* w,
                    const double* theta, const double* phi, int* z,
                    uint64_t seed, uint32_t iter) {
  double* pmf = (double*)malloc(sizeof(double) * (size_t)K);
  for (int d = 0; d < D; ++d) {
    const double* th = theta + (size_t)d * K;
    for (int t = doc_off[d]; t < doc_off[d + 1]; ++t) {
      for (int k = 0; k < K; ++k) {
        double prob = 1.0;
        prob *= th[k];
        prob *= phi[(size_t)k * V + w[t]];
        pmf[k] = prob;
      }
      orc_stream s = orc_make(seed, (uint32_t)t, iter, ORC_TAG_Z);
      z[t] = orc_unnorm_disc(&s, pmf, K);
    }
  }
  free(pmf);
}

/* conj_stat, CgConj.hs:171-177 after the reset of CgKern.hs:103-107. */
void orc_lda_conj_stat(int D, int K, int V, const int* doc_off, const int* w,
                       const int* z, int* cnt_dk, int* cnt_kw) {
  memset(cnt_dk, 0, sizeof(int) * (size_t)D * K);
  memset(cnt_kw, 0, sizeof(int) * (size_t)K * V);
  for (int d = 0; d < D; ++d)
    for (int t = doc_off[d]; t < doc_off[d + 1]; ++t) {
      cnt_dk[(size_t)d * K + z[t]] += 1;
      cnt_kw[(size_t)z[t] * V + w[t]] += 1;
    }
}

/* Dirichlet-Categorical conjugate draw per row, cbits/augur_dist.c:526-538:
 * gamma(alpha_i + cnt_i, 1) per element, sequential sum, divide.  Element
 * substream (row*cols + i, iter, tag). */
void orc_dirichlet_rows(int rows, int cols, const double* alpha, const int* cnt,
                        double* out, uint64_t seed, uint32_t iter, uint32_t tag) {
  for (int r = 0; r < rows; ++r) {
    double* dst = out + (size_t)r * cols;
    double acc = 0.0;
    for (int i = 0; i < cols; ++i) {
      orc_stream s = orc_make(seed, (uint32_t)((size_t)r * cols + i), iter, tag);
      double g = orc_gamma(&s, alpha[i] + (double)cnt[(size_t)r * cols + i], 1.0);
      dst[i] = g;
      acc += g;
    }
    for (int i = 0; i < cols; ++i) dst[i] = dst[i] / acc;
  }
}

void orc_lda_conj_theta(int D, int K, const double* alpha, const int* cnt_dk,
                        double* theta, uint64_t seed, uint32_t iter) {
  orc_dirichlet_rows(D, K, alpha, cnt_dk, theta, seed, iter, ORC_TAG_THETA);
}

void orc_lda_conj_phi(int K, int V, const double* beta, const int* cnt_kw,
                      double* phi, uint64_t seed, uint32_t iter) {
  orc_dirichlet_rows(K, V, beta, cnt_kw, phi, seed, iter, ORC_TAG_PHI);
}

/* augur_step for ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z],
 * CgKern.hs:144-178. */
void orc_lda_sweeps(int D, int K, int V, const int* doc_off, const int* w,
                    const double* alpha, const double* beta, double* theta,
                    double* phi, int* z, int* cnt_dk, int* cnt_kw,
                    uint64_t seed, uint32_t iter0, int n_sweeps) {
  for (int s = 0; s < n_sweeps; ++s) {
    uint32_t it = iter0 + (uint32_t)s;
    orc_lda_conj_stat(D, K, V, doc_off, w, z, cnt_dk, cnt_kw);
    orc_lda_conj_theta(D, K, alpha, cnt_dk, theta, seed, it);
    orc_lda_conj_phi(K, V, beta, cnt_kw, phi, seed, it);
    orc_lda_disc_z(D, K, V, doc_off, w, theta, phi, z, seed, it);
  }
}

/* ------------------------------------------------------------------------
 * Hierarchical logistic regression (compiler/augur/test/hlr.rv and the
 * InvGamma-variance variant without bias):
 *   v ~ Exponential(lam) | InvGamma(a0, s0);  b ~ Normal(0, v) (optional);
 *   theta[k] ~ Normal(0, v);  y[n] ~ Bernoulli(sigmoid(theta . x[n] + b)),
 * and the same priors with the other generalised-linear likelihoods the
 * reference's modelling language can state with t = theta . x[n] + b
 * (lik): 1 y[n] ~ Poisson(exp(t)) (augur_poisson_ll, cbits/augur_dist.c:
 * 124-130), 2 yr[n] ~ Normal(t, obs_var) with a fixed variance
 * (augur_normal_ll, :372-381).
 * Parameters are one vector par = [theta[0..D-1], b, v].  A block is a list
 * of indices into par in the schedule's order (HMC [v, b, theta] -> D+1, D,
 * 0..D-1).  `compat` selects the reference's own density formulas
 * (cbits/augur_dist.c:59-72,231-247,345-394), including its Normal log
 * density -log(var) - t^2/(2 var) and its dNormal/dvar of -var/2 + ...;
 * compat = 0 uses the textbook densities with numerically stable logistic
 * terms.
 * --------------------------------------------------------------------- */
#define ORC_LARGE 1e8
typedef struct {
  int N, D, has_b, vprior, compat; /* vprior: 0 Exponential(lam), 1 InvGamma(a0, s0) */
  double lam, a0, s0;
  const double* X; /* N x D row-major */
  const int* y;    /* Bernoulli and Poisson labels */
  int lik;         /* 0 Bernoulli(sigmoid(t)), 1 Poisson(exp(t)), 2 Normal(t, obs_var) */
  double obs_var;
  const double* yr; /* Normal labels */
} orc_hlr;

static double orc_expit(double x) { return 1.0 / (1.0 + exp(-x)); }

static double orc_normal_ll(const orc_hlr* m, double pt, double mean, double var) {
  if (m->compat) {
    if (var > 0.0) { double t = pt - mean; return (-log(var)) - (0.5 * t * t / var); }
    return -ORC_LARGE;
  }
  if (!(var > 0.0)) return -INFINITY;
  double t = pt - mean;
  return -0.5 * log(2.0 * 3.14159265358979323846 * var) - 0.5 * t * t / var;
}
static double orc_normal_dotpt(double pt, double mean, double var) { return -(pt - mean) / var; }
static double orc_normal_dotarg2(const orc_hlr* m, double pt, double mean, double var) {
  double t = pt - mean;
  if (m->compat) return (-0.5 * var) + (0.5 * (t * t) / (var * var));
  return (-0.5 / var) + (0.5 * (t * t) / (var * var));
}
static double orc_vprior_ll(const orc_hlr* m, double v) {
  if (m->vprior == 0) {                     /* augur_exponential_ll, augur_dist.c:231-238 */
    if (m->lam > 0.0 && v > 0.0) return log(m->lam) - m->lam * v;
    return m->compat ? -ORC_LARGE : -INFINITY;
  }
  if (!(v > 0.0)) return m->compat ? -ORC_LARGE : -INFINITY;  /* augur_invgamma_ll :345-347 */
  return m->a0 * log(m->s0) - lgamma(m->a0) - (m->a0 + 1.0) * log(v) - m->s0 / v;
}
static double orc_vprior_dot(const orc_hlr* m, double v) {
  if (m->vprior == 0) return (m->lam > 0.0 && v > 0.0) ? -m->lam : 0.0;   /* :240-246 */
  return -(m->a0 + 1.0) / v + m->s0 / (v * v);                             /* :349-351 */
}

/* Data factor of one row: log Bern(y | sigmoid(t)) and d/dt of it. */
static double orc_bern_ll(const orc_hlr* m, int y, double t) {
  if (m->compat) {                          /* augur_bernoulli_ll(y, augur_expit(t)) */
    double p = orc_expit(t);
    if (p >= 0.0 && p <= 1.0) return log(y * p + (1 - y) * (1.0 - p));
    return -ORC_LARGE;
  }
  double sp = (t > 0 ? t : 0.0) + log1p(exp(-fabs(t)));   /* softplus */
  return y ? t - sp : -sp;
}
static double orc_bern_dt(const orc_hlr* m, int y, double t) {
  if (m->compat) {                          /* dotarg1 (:68-71) x expit_grad_0 (augur_math.c:56-59) */
    double p = orc_expit(t);
    double denom = (y * p + (1 - y) * (1.0 - p));
    double adj3 = (y + y - 1) / denom;
    double e = orc_expit(t);
    return adj3 * (e * (1.0 - e));
  }
  return (double)y - orc_expit(t);
}

/* Poisson(exp(t)): the reference's y log(rate) - rate - sum_{k <= y} log k
 * and its adjoint through exp, augur_poisson_dotarg1 (:132-139) x exp(t);
 * compat = 0: y t - exp(t) - lgamma(y + 1) and y - exp(t). */
static double orc_pois_ll(const orc_hlr* m, int y, double t) {
  if (m->compat) {
    const double rate = exp(t);
    double acc = 0.0;
    for (int k = 1; k <= y; k++) acc += log((double)k);
    return y * log(rate) - rate - acc;
  }
  return y * t - exp(t) - lgamma(y + 1.0);
}
static double orc_pois_dt(const orc_hlr* m, int y, double t) {
  const double rate = exp(t);
  if (m->compat) return (rate > 0.0 ? y / rate - 1.0 : -ORC_LARGE) * rate;
  return y - rate;
}

/* Data factor of row n at t and its derivative, by likelihood. */
static double orc_lik_ll(const orc_hlr* m, int n, double t) {
  if (m->lik == 1) return orc_pois_ll(m, m->y[n], t);
  if (m->lik == 2) return orc_normal_ll(m, m->yr[n], t, m->obs_var);
  return orc_bern_ll(m, m->y[n], t);
}
static double orc_lik_dt(const orc_hlr* m, int n, double t) {
  if (m->lik == 1) return orc_pois_dt(m, m->y[n], t);
  if (m->lik == 2) return (m->yr[n] - t) / m->obs_var;   /* augur_normal_dotarg1, :388-390 */
  return orc_bern_dt(m, m->y[n], t);
}

static int orc_in_block(const int* idx, int P, int lo, int hi) {
  for (int j = 0; j < P; ++j) if (idx[j] >= lo && idx[j] < hi) return 1;
  return 0;
}

/* Full conditional of the block (CgLike.hs:139-147,254-258): factors that
 * mention a block variable, in model order, each Pi factor a sequential
 * sum over its index, accumulated onto ll = 0. */
double orc_hlr_ll(const orc_hlr* m, const double* par, const int* idx, int P) {
  const int D = m->D;
  const double b = m->has_b ? par[D] : 0.0, v = par[D + 1];
  const int in_th = orc_in_block(idx, P, 0, D);
  const int in_b = m->has_b && orc_in_block(idx, P, D, D + 1);
  const int in_v = orc_in_block(idx, P, D + 1, D + 2);
  double ll = 0.0;
  if (in_v) ll += orc_vprior_ll(m, v);
  if (m->has_b && (in_b || in_v)) ll += orc_normal_ll(m, b, 0.0, v);
  if (in_th || in_v) {
    double s = 0.0;
    for (int k = 0; k < D; ++k) s += orc_normal_ll(m, par[k], 0.0, v);
    ll += s;
  }
  if (in_th || in_b) {
    double s = 0.0;
    for (int n = 0; n < m->N; ++n) {
      const double* x = m->X + (size_t)n * D;
      double dot = 0.0;
      for (int k = 0; k < D; ++k) dot += par[k] * x[k];
      s += orc_lik_ll(m, n, dot + b);
    }
    ll += s;
  }
  return ll;
}

/* Gradient of orc_hlr_ll with respect to the block (CgGrad.hs:165-376):
 * adjoints start at zero; factors in model order; the data factor adds
 * adj_t * x[n] per row in row order. */
void orc_hlr_grad(const orc_hlr* m, const double* par, const int* idx, int P, double* g) {
  const int D = m->D;
  const double b = m->has_b ? par[D] : 0.0, v = par[D + 1];
  double* full = (double*)calloc((size_t)D + 2, sizeof(double));
  const int in_th = orc_in_block(idx, P, 0, D);
  const int in_b = m->has_b && orc_in_block(idx, P, D, D + 1);
  const int in_v = orc_in_block(idx, P, D + 1, D + 2);
  if (in_v) full[D + 1] += orc_vprior_dot(m, v);
  if (m->has_b && (in_b || in_v)) {
    if (in_b) full[D] += orc_normal_dotpt(b, 0.0, v);
    if (in_v) full[D + 1] += orc_normal_dotarg2(m, b, 0.0, v);
  }
  if (in_th || in_v) {
    for (int k = 0; k < D; ++k) {
      if (in_th) full[k] += orc_normal_dotpt(par[k], 0.0, v);
      if (in_v) full[D + 1] += orc_normal_dotarg2(m, par[k], 0.0, v);
    }
  }
  if (in_th || in_b) {
    for (int n = 0; n < m->N; ++n) {
      const double* x = m->X + (size_t)n * D;
      double dot = 0.0;
      for (int k = 0; k < D; ++k) dot += par[k] * x[k];
      double r = orc_lik_dt(m, n, dot + b);
      if (in_b) full[D] += r;
      if (in_th) for (int k = 0; k < D; ++k) full[k] += r * x[k];
    }
  }
  for (int j = 0; j < P; ++j) g[j] = full[idx[j]];
  free(full);
}

/* Batched helper for parity tests: ll and gradient for C parameter vectors. */
void orc_hlr_ll_grad_batch(const orc_hlr* m, int C, const double* pars, const int* idx, int P,
                           double* ll, double* g) {
  for (int c = 0; c < C; ++c) {
    const double* par = pars + (size_t)c * (m->D + 2);
    ll[c] = orc_hlr_ll(m, par, idx, P);
    orc_hlr_grad(m, par, idx, P, g + (size_t)c * P);
  }
}

/* ---- HMC: cbits/augur_mcmclib.h:343-424 (h_augur_mcmc_leapfrog, _hmc) ----
 * Substreams: momentum element j of chain c: (c*P + j, iter, MOM|comp<<8);
 * jitter and accept: (c, iter, HMC|comp<<8) positions 0, 1 (jitter), 2
 * (accept u).  `simsteps_out` reports L; returns 1 on accept. */
static void orc_set_block(double* par, const int* idx, int P, const double* q) {
  for (int j = 0; j < P; ++j) par[idx[j]] = q[j];
}
static void orc_get_block(const double* par, const int* idx, int P, double* q) {
  for (int j = 0; j < P; ++j) q[j] = par[idx[j]];
}

int orc_hlr_hmc(const orc_hlr* m, double* par, const int* idx, int P, double simlen, double eps,
                uint64_t seed, uint32_t iter, uint32_t chain, uint32_t comp, int* simsteps_out,
                double* prop_out) {
  const int NP = m->D + 2;
  double* p0 = (double*)malloc(sizeof(double) * P);
  double* ps = (double*)malloc(sizeof(double) * P);
  double* g = (double*)malloc(sizeof(double) * P);
  double* th0 = (double*)malloc(sizeof(double) * P);
  double* ths = (double*)malloc(sizeof(double) * P);
  double* prop = (double*)malloc(sizeof(double) * NP);
  for (int j = 0; j < P; ++j) {
    orc_stream s = orc_make(seed, chain * (uint32_t)P + j, iter, ORC_TAG_MOM | (comp << 8));
    p0[j] = orc_normal(&s);
  }
  orc_stream h = orc_make(seed, chain, iter, ORC_TAG_HMC | (comp << 8));
  double scale_eps = 0.8 + orc_uniform(&h) * (1.2 - 0.8);
  double stepsize = scale_eps * eps;
  double sj = 0.9 + orc_uniform(&h) * (1.1 - 0.9);
  /* augur_max is unsigned (cbits/augur_util.c:61-64) */
  unsigned rl = (unsigned)round(sj * simlen / stepsize);
  int simsteps = (int)(rl > 1u ? rl : 1u);
  memcpy(prop, par, sizeof(double) * NP);
  orc_get_block(par, idx, P, th0);
  memcpy(ths, th0, sizeof(double) * P);
  /* leapfrog (:343-375) */
  orc_hlr_grad(m, par, idx, P, g);
  for (int j = 0; j < P; ++j) ps[j] = p0[j] + stepsize / 2.0 * g[j];
  for (int l = 0; l < simsteps; ++l) {
    for (int j = 0; j < P; ++j) ths[j] = ths[j] + stepsize * ps[j];
    orc_set_block(prop, idx, P, ths);
    if (l != simsteps - 1) {
      orc_hlr_grad(m, prop, idx, P, g);
      for (int j = 0; j < P; ++j) ps[j] = ps[j] + stepsize * g[j];
    }
  }
  orc_hlr_grad(m, prop, idx, P, g);
  for (int j = 0; j < P; ++j) ps[j] = ps[j] + stepsize / 2.0 * g[j];
  double k0 = 0.0, k1 = 0.0;
  for (int j = 0; j < P; ++j) k0 += p0[j] * p0[j];
  for (int j = 0; j < P; ++j) k1 += ps[j] * ps[j];
  double auxll = k0 / 2.0 - k1 / 2.0;
  /* augur_mcmc_ar (:70-83) */
  double currll = orc_hlr_ll(m, par, idx, P);
  double propll = orc_hlr_ll(m, prop, idx, P);
  double u = orc_uniform(&h);
  int acc = log(u) < propll - currll + auxll;
  if (prop_out) memcpy(prop_out, prop, sizeof(double) * NP);
  if (acc) memcpy(par, prop, sizeof(double) * NP);
  if (simsteps_out) *simsteps_out = simsteps;
  free(p0); free(ps); free(g); free(th0); free(ths); free(prop);
  return acc;
}

/* ---- Reflective slice: cbits/augur_mcmclib.h:498-543 (h_augur_mcmc_refl_slice)
 * Momentum p0 ~ N(0, I) from (c*P + j, iter, MOM|comp<<8); the slice level
 * z = ll(curr) - Exp(1) with the exponential from (c, iter, RSLICE|comp<<8);
 * simsteps = augur_max(1, round(simlen / eps)) (unsigned); each step moves
 * the block by eps * p0 and, if the point left the slice (ll < z), reflects
 * p0 off the gradient there: p0 += (-2 (p0.g)/(g.g)) g.  The move is kept
 * only if the last point is inside the slice.  Returns 1 on a move;
 * `reflections_out` counts the reflections. */
int orc_hlr_rslice(const orc_hlr* m, double* par, const int* idx, int P, double simlen, double eps,
                   uint64_t seed, uint32_t iter, uint32_t chain, uint32_t comp, int* simsteps_out,
                   int* reflections_out) {
  const int NP = m->D + 2;
  double* p0 = (double*)malloc(sizeof(double) * P);
  double* g = (double*)malloc(sizeof(double) * P);
  double* ths = (double*)malloc(sizeof(double) * P);
  double* prop = (double*)malloc(sizeof(double) * NP);
  for (int j = 0; j < P; ++j) {
    orc_stream s = orc_make(seed, chain * (uint32_t)P + j, iter, ORC_TAG_MOM | (comp << 8));
    p0[j] = orc_normal(&s);
  }
  orc_stream h = orc_make(seed, chain, iter, ORC_TAG_RSLICE | (comp << 8));
  const double z = orc_hlr_ll(m, par, idx, P) - (-1.0 * log(orc_uniform(&h)));
  const double stepsize = eps;
  unsigned rl = (unsigned)round(simlen / stepsize);
  const int simsteps = (int)(rl > 1u ? rl : 1u);
  memcpy(prop, par, sizeof(double) * NP);
  orc_get_block(par, idx, P, ths);
  int cond = 0, refl = 0;
  for (int i = 0; i < simsteps; ++i) {
    for (int j = 0; j < P; ++j) ths[j] = ths[j] + stepsize * p0[j];
    orc_set_block(prop, idx, P, ths);
    cond = orc_hlr_ll(m, prop, idx, P) < z;
    if (cond) {
      orc_hlr_grad(m, prop, idx, P, g);
      double a1 = 0.0, a2 = 0.0;
      for (int j = 0; j < P; ++j) a1 += p0[j] * g[j];
      for (int j = 0; j < P; ++j) a2 += g[j] * g[j];
      const double scale = a1 / a2;
      for (int j = 0; j < P; ++j) p0[j] = p0[j] + (-2.0 * scale) * g[j];
      ++refl;
    }
  }
  if (!cond) memcpy(par, prop, sizeof(double) * NP);
  if (simsteps_out) *simsteps_out = simsteps;
  if (reflections_out) *reflections_out = refl;
  free(p0); free(g); free(ths); free(prop);
  return !cond;
}

/* ---- NUTS: cbits/augur_mcmclib.h:575-776, restated with its exact control
 * flow (two gradients per leaf, the stacks of augur_blkstk.c, the subtree
 * endpoints taken from the most recent j == 1 push, the proposal kept only
 * if the final doubling accepted one).  deltaMax = 1000 (:152).  Substreams:
 * momentum (c*P + j, iter, MOM|comp<<8); every other draw sequentially from
 * (c, iter, NUTS|comp<<8): exponential slice, then per doubling the
 * direction coin, the subtree coins in recursion order, the outer coin. */
#define ORC_STK_MAX 16
typedef struct {
  double* b[ORC_STK_MAX];
  int hd;
} orc_stk;

typedef struct {
  const orc_hlr* m;
  const int* idx;
  int P;
  double* mod;      /* full parameter vector whose block is the working theta */
  double* g;
  double stepsize, logu;
  orc_stream* h;
  orc_stk tp, ts, ms; /* theta_prop, theta, mom stacks */
  double* work;
  int overflow, leaves;
} orc_nuts;

static void orc_push(orc_nuts* t, orc_stk* s, const double* v) {
  s->hd++;
  if (s->hd >= ORC_STK_MAX) { t->overflow = 1; s->hd = ORC_STK_MAX - 1; return; }
  memcpy(s->b[s->hd], v, sizeof(double) * t->P);
}
static double* orc_pop(orc_stk* s) { double* r = s->b[s->hd < 0 ? 0 : s->hd]; s->hd--; return r; }
static double* orc_peek(orc_stk* s) { return s->b[s->hd < 0 ? 0 : s->hd]; }

static double orc_dot(const double* a, const double* b, int P) {
  double acc = 0.0;
  for (int j = 0; j < P; ++j) acc += a[j] * b[j];
  return acc;
}

static int orc_update_s(const orc_nuts* t, int s, const double* tp, const double* mp,
                        const double* tm, const double* mm) {
  if (s == 1) {
    for (int j = 0; j < t->P; ++j) t->work[j] = tp[j] + -1.0 * tm[j];
    int ut1 = orc_dot(t->work, mp, t->P) >= 0.0;
    int ut2 = orc_dot(t->work, mm, t->P) >= 0.0;
    if (ut1 && ut2) return 1;
  }
  return 0;
}

static void orc_leapfrog1(orc_nuts* t, double* theta, double* mom) {
  const int P = t->P;
  const double s = t->stepsize;
  orc_set_block(t->mod, t->idx, P, theta);
  orc_hlr_grad(t->m, t->mod, t->idx, P, t->g);
  for (int j = 0; j < P; ++j) mom[j] = mom[j] + s / 2.0 * t->g[j];
  for (int j = 0; j < P; ++j) theta[j] = theta[j] + s * mom[j];
  orc_set_block(t->mod, t->idx, P, theta);
  orc_hlr_grad(t->m, t->mod, t->idx, P, t->g);
  for (int j = 0; j < P; ++j) mom[j] = mom[j] + s / 2.0 * t->g[j];
}

typedef struct { int n, s; } orc_nret;

static orc_nret orc_build(orc_nuts* t, double* theta, double* mom, int j, int dir) {
  orc_nret r;
  if (j == 0) {
    orc_leapfrog1(t, theta, mom);
    t->leaves++;
    orc_push(t, &t->tp, theta);
    double ll = orc_hlr_ll(t->m, t->mod, t->idx, t->P) - 0.5 * orc_dot(mom, mom, t->P);
    r.n = t->logu <= ll;
    r.s = t->logu < 1000.0 + ll;
    return r;
  }
  orc_nret left = orc_build(t, theta, mom, j - 1, dir);
  if (left.s == 1) {
    if (j == 1) { orc_push(t, &t->ts, theta); orc_push(t, &t->ms, mom); }
    orc_nret right = orc_build(t, theta, mom, j - 1, dir);
    double* p1 = orc_pop(&t->tp);
    double* p2 = orc_pop(&t->tp);
    double bias = ((double)right.n) / (left.n + right.n);
    if (!(orc_uniform(t->h) < bias)) orc_push(t, &t->tp, p2);
    else orc_push(t, &t->tp, p1);
    left.n += right.n;
    const double *tp, *mp, *tm, *mm;
    if (dir == 0) { tp = orc_peek(&t->ts); mp = orc_peek(&t->ms); tm = theta; mm = mom; }
    else { tm = orc_peek(&t->ts); mm = orc_peek(&t->ms); tp = theta; mp = mom; }
    left.s = orc_update_s(t, right.s, tp, mp, tm, mm);
    if (j > 1) { orc_pop(&t->ts); orc_pop(&t->ms); }
  }
  return left;
}

/* Returns the number of doublings; *leaves_out the leapfrog leaves; 
 * *overflow_out = 1 if a stack passed the reference's 16 entries (the
 * reference's behaviour is then undefined). */
int orc_hlr_nuts(const orc_hlr* m, double* par, const int* idx, int P, double eps, uint64_t seed,
                 uint32_t iter, uint32_t chain, uint32_t comp, int max_depth, int* leaves_out,
                 int* overflow_out) {
  const int NP = m->D + 2;
  orc_nuts t;
  memset(&t, 0, sizeof(t));
  t.m = m; t.idx = idx; t.P = P;
  double* mem = (double*)calloc((size_t)P * (3 * ORC_STK_MAX + 7) + NP, sizeof(double));
  double* th0 = mem; double* thm = th0 + P; double* mm = thm + P; double* thp = mm + P;
  double* mp = thp + P; double* thprop = mp + P; t.work = thprop + P;
  t.g = t.work + P; t.mod = t.g + P;
  double* sb = t.mod + NP;
  for (int i = 0; i < ORC_STK_MAX; ++i) {
    t.tp.b[i] = sb + (size_t)(3 * i) * P;
    t.ts.b[i] = sb + (size_t)(3 * i + 1) * P;
    t.ms.b[i] = sb + (size_t)(3 * i + 2) * P;
  }
  t.tp.hd = t.ts.hd = t.ms.hd = -1;
  memcpy(t.mod, par, sizeof(double) * NP);
  orc_get_block(par, idx, P, th0);
  memcpy(thm, th0, sizeof(double) * P);
  for (int j = 0; j < P; ++j) {
    orc_stream s = orc_make(seed, chain * (uint32_t)P + j, iter, ORC_TAG_MOM | (comp << 8));
    mm[j] = orc_normal(&s);
  }
  memcpy(thp, th0, sizeof(double) * P);
  memcpy(mp, mm, sizeof(double) * P);
  orc_stream h = orc_make(seed, chain, iter, ORC_TAG_NUTS | (comp << 8));
  t.h = &h;
  double e = -1.0 * log(orc_uniform(&h));
  t.logu = orc_hlr_ll(m, par, idx, P) - 0.5 * orc_dot(mm, mm, P) - e;
  int n = 1, j = 0, s = 1;
  for (;;) {
    int f_cpy = 0;
    orc_nret r;
    t.ts.hd = -1; t.ms.hd = -1;
    if (orc_uniform(&h) < 0.5) {
      t.stepsize = -eps;
      memcpy(thprop, thm, sizeof(double) * P);
      r = orc_build(&t, thprop, mm, j, 0);
      memcpy(thm, thprop, sizeof(double) * P);
    } else {
      t.stepsize = eps;
      memcpy(thprop, thp, sizeof(double) * P);
      r = orc_build(&t, thprop, mp, j, 1);
      memcpy(thp, thprop, sizeof(double) * P);
    }
    double* pp = orc_pop(&t.tp);
    if (r.s == 1) {
      /* augur_min takes and returns unsigned int (cbits/augur_util.c:56-59),
       * so the ratio is truncated: the bias is 1 when n' >= n, else 0. */
      unsigned ratio = (unsigned)(((double)r.n) / n);
      double bias = (double)(ratio < 1u ? ratio : 1u);
      if (orc_uniform(&h) < bias) { memcpy(thprop, pp, sizeof(double) * P); f_cpy = 1; }
    }
    n += r.n;
    s = orc_update_s(&t, r.s, thp, mp, thm, mm);
    j += 1;
    if (s != 1 || j >= max_depth || t.overflow) {
      if (f_cpy) memcpy(th0, thprop, sizeof(double) * P);
      break;
    }
  }
  orc_set_block(par, idx, P, th0);
  if (leaves_out) *leaves_out = t.leaves;
  if (overflow_out) *overflow_out = t.overflow;
  free(mem);
  return j;
}

/* ---- MWG on a scalar of par: cbits/augur_mcmclib.h:89-105,178-193 with
 * the generated prop_/swap_ of CgUserProp.hs:131-210.  Proposal
 * Normal(x, var); compat uses the generated log-correction
 * ll(x; x, var) - ll(x'; x, var) (both evaluated at the current state);
 * otherwise the symmetric random walk's correction 0.  Substream
 * (c, iter, MWG|comp<<8): normal, then the accept uniform. */
int orc_hlr_mwg(const orc_hlr* m, double* par, int which, double var, uint64_t seed,
                uint32_t iter, uint32_t chain, uint32_t comp) {
  const int NP = m->D + 2;
  double* prop = (double*)malloc(sizeof(double) * NP);
  memcpy(prop, par, sizeof(double) * NP);
  orc_stream s = orc_make(seed, chain, iter, ORC_TAG_MWG | (comp << 8));
  const double x = par[which];
  const double xp = x + sqrt(var) * orc_normal(&s);
  prop[which] = xp;
  double corr = 0.0;
  if (m->compat) corr = orc_normal_ll(m, x, x, var) - orc_normal_ll(m, xp, x, var);
  int idx[1] = {which};
  double currll = orc_hlr_ll(m, par, idx, 1);
  double propll = orc_hlr_ll(m, prop, idx, 1);
  double u = orc_uniform(&s);
  int acc = log(u) < propll - currll + corr;
  if (acc) par[which] = xp;
  free(prop);
  return acc;
}

/* ------------------------------------------------------------------------
 * Gaussian mixtures (compiler/augur/test/mvgmm.rv, hmvgmm.rv).
 * Square d x d row-major matrices, operations restated from
 * cbits/augur_matop.c:312-420 and the samplers of cbits/augur_dist.c:543-757,
 * each with the reference's loop order.
 * --------------------------------------------------------------------- */
#define M_(A, i, j) (A)[(size_t)(i) * d + (j)]

/* augur_mat_cholesky (:312-328): lower factor in place, upper unchanged. */
void orc_mat_cholesky(double* A, int d) {
  for (int i = 0; i < d; i++)
    for (int j = 0; j < i + 1; j++) {
      double s = 0.0;
      for (int k = 0; k < j; k++) s += M_(A, i, k) * M_(A, j, k);
      if (i == j) M_(A, i, j) = sqrt(M_(A, i, i) - s);
      else M_(A, i, j) = 1.0 / M_(A, j, j) * (M_(A, i, j) - s);
    }
}

/* augur_mat_lower_trmi (:335-345). */
void orc_mat_lower_trmi(double* L, int d) {
  for (int c = 0; c < d; c++)
    for (int m = 0; m < d; m++) {
      double b = (c == m) ? 1.0 : 0.0;
      for (int i = 0; i < m; i++) b -= M_(L, m, i) * M_(L, i, c);
      M_(L, m, c) = b / M_(L, m, m);
    }
}

/* augur_mat_cholesky_invert (:363-375) with augur_mat_lower_trtcpy (:351-357). */
void orc_mat_cholesky_invert(double* A, int d) {
  orc_mat_lower_trmi(A, d);
  for (int c = 0; c < d; c++)
    for (int r = c; r < d; r++) {
      double acc = 0.0;
      for (int k = c; k < d; k++) acc += M_(A, k, r) * M_(A, k, c);
      M_(A, r, c) = acc;
    }
  for (int c = 0; c < d; c++)
    for (int r = c + 1; r < d; r++) M_(A, c, r) = M_(A, r, c);
}

/* augur_mat_trtrmm (:381-392): L2 = L1 L2. */
static void orc_mat_trtrmm(const double* L1, double* L2, int d) {
  for (int i = d; i > 0 && i--;) {
    for (int j = 0; j < d; j++) {
      double tmp = 0.0;
      for (int k = 0; k < i; k++) tmp += M_(L1, i, k) * M_(L2, k, j);
      tmp += M_(L1, i, i) * M_(L2, i, j);
      M_(L2, i, j) = tmp;
    }
  }
}

/* augur_mat_trvm (:398-406): v = L v. */
static void orc_mat_trvm(const double* L, double* v, int d) {
  for (int i = d - 1; i >= 0; i--) {
    double tmp = 0.0;
    for (int j = 0; j <= i; j++) tmp += M_(L, i, j) * v[j];
    v[i] = tmp;
  }
}

/* augur_mat_mvm (:412-420): dst = A v. */
static void orc_mat_mvm(double* dst, const double* A, const double* v, int d) {
  for (int i = 0; i < d; i++) {
    double tmp = 0.0;
    for (int j = 0; j < d; j++) tmp += M_(A, i, j) * v[j];
    dst[i] = tmp;
  }
}

/* augur_mvnormal_ll (augur_dist.c:548-568). */
double orc_mvnormal_ll(const double* pt, const double* mean, const double* cov, int d) {
  double* L = (double*)malloc(sizeof(double) * d * d);
  double* w = (double*)malloc(sizeof(double) * d);
  for (int i = 0; i < d; i++) w[i] = pt[i] - mean[i];
  memcpy(L, cov, sizeof(double) * d * d);
  orc_mat_cholesky(L, d);
  double det = 1.0;
  for (int i = 0; i < d; i++) det *= M_(L, i, i);
  det *= det;
  orc_mat_lower_trmi(L, d);
  orc_mat_trvm(L, w, d);
  double expon = 0.0;
  for (int i = 0; i < d; i++) expon += w[i] * w[i];
  double c = -0.5 * ((double)d) * log(2.0 * 3.14159265358979323846264338327950288);
  free(L); free(w);
  return c - 0.5 * log(det) - 0.5 * expon;
}

/* augur_mvnormal_sample (:622-630): result = chol(cov) z + mean. */
static void orc_mvnormal_sample(orc_stream* s, double* result, const double* mean, const double* cov, int d) {
  double* L = (double*)malloc(sizeof(double) * d * d);
  for (int i = 0; i < d; i++) result[i] = orc_normal(s);
  memcpy(L, cov, sizeof(double) * d * d);
  orc_mat_cholesky(L, d);
  orc_mat_trvm(L, result, d);
  for (int i = 0; i < d; i++) result[i] = result[i] + mean[i];
  free(L);
}

/* augur_mvnormal_mvnormal_conj (:633-669).  `sum` is scaled in place by
 * 1/cnt as in the reference. */
static void orc_mvn_mvn_conj(orc_stream* s, double* result, const double* mu0, const double* cov0,
                             double* sum, int cnt, const double* cov, int d) {
  double* L0 = (double*)malloc(sizeof(double) * d * d);
  double* L = (double*)malloc(sizeof(double) * d * d);
  double* w0 = (double*)malloc(sizeof(double) * d);
  double* mean = (double*)malloc(sizeof(double) * d);
  memcpy(L0, cov0, sizeof(double) * d * d);
  orc_mat_cholesky(L0, d);
  orc_mat_cholesky_invert(L0, d);
  memcpy(L, cov, sizeof(double) * d * d);
  orc_mat_cholesky(L, d);
  orc_mat_cholesky_invert(L, d);
  for (int i = 0; i < d * d; i++) L[i] = cnt * L[i];             /* augur_mat_ms */
  orc_mat_mvm(result, L0, mu0, d);
  double sc = cnt == 0 ? 1.0 : 1.0 / cnt;                         /* augur_vec_scale */
  for (int i = 0; i < d; i++) sum[i] = sc * sum[i];
  orc_mat_mvm(w0, L, sum, d);
  for (int i = 0; i < d; i++) result[i] = result[i] + w0[i];
  for (int i = 0; i < d * d; i++) L0[i] = L0[i] + L[i];           /* augur_mat_plus */
  orc_mat_cholesky(L0, d);
  orc_mat_cholesky_invert(L0, d);
  orc_mat_mvm(mean, L0, result, d);
  orc_mvnormal_sample(s, result, mean, L0, d);
  free(L0); free(L); free(w0); free(mean);
}

/* bartlett_decomp (:722-738) with augur_chisquared_sample (:213-220). */
static void orc_bartlett(orc_stream* s, int n, double* A, int d) {
  for (int i = 0; i < d; i++)
    for (int j = 0; j < d; j++) {
      if (j < i) M_(A, i, j) = orc_normal(s);
      else if (j > i) M_(A, i, j) = 0.0;
      else {
        double chi = 0.0;
        for (int t = 0; t < n - i; t++) { double z = orc_normal(s); chi += z * z; }
        M_(A, i, j) = sqrt(chi);
      }
    }
}

/* augur_invwishart_sample (:740-749). */
static void orc_invwishart_sample(orc_stream* s, double* result, int df, const double* scale, int d) {
  double* L = (double*)malloc(sizeof(double) * d * d);
  memcpy(L, scale, sizeof(double) * d * d);
  orc_mat_cholesky(L, d);
  orc_mat_cholesky_invert(L, d);
  orc_mat_cholesky(L, d);
  orc_bartlett(s, df, result, d);
  orc_mat_trtrmm(L, result, d);
  orc_mat_cholesky_invert(result, d);
  free(L);
}

/* Dirichlet-Categorical conjugate draw of a K-vector (augur_dist.c:526-538),
 * element substream (k, iter, tag). */
static void orc_dirichlet_vec(int K, const double* alpha, const int* cnt, double* out, uint64_t seed,
                              uint32_t iter, uint32_t tag) {
  orc_dirichlet_rows(1, K, alpha, cnt, out, seed, iter, tag);
}

typedef struct {
  int N, d, K, shared_cov;     /* shared_cov: mvgmm (one covs); else hmvgmm cov[K] */
  const double* Y;             /* N x d */
  const double* mu0;           /* d */
  const double* cov0;          /* d x d */
  const double* alpha;         /* K (hmvgmm) */
  int df;                      /* InvWishart df (hmvgmm) */
  const double* scale0;        /* d x d (hmvgmm) */
} orc_gmm;

/* disc_z (CgDisc.hs:122-156): pmf[k] = (1 * pis[k]) * mvnormal_pdf(y, mu[k],
 * cov[k]) (augur_mvnormal_pdf = exp(ll)), then augur_unnorm_disc_samp.
 * Substream (n, iter, Z). */
void orc_gmm_disc_z(const orc_gmm* g, const double* pis, const double* mu, const double* cov,
                    int* z, uint64_t seed, uint32_t iter) {
  const int d = g->d, K = g->K;
  double* pmf = (double*)malloc(sizeof(double) * K);
  for (int n = 0; n < g->N; n++) {
    for (int k = 0; k < K; k++) {
      const double* ck = g->shared_cov ? cov : cov + (size_t)k * d * d;
      double prob = 1.0;
      prob *= pis[k];
      prob *= exp(orc_mvnormal_ll(g->Y + (size_t)n * d, mu + (size_t)k * d, ck, d));
      pmf[k] = prob;
    }
    orc_stream s = orc_make(seed, (uint32_t)n, iter, ORC_TAG_Z);
    z[n] = orc_unnorm_disc(&s, pmf, K);
  }
  free(pmf);
}

/* The same draw for the listed points only: z_out[i] is the assignment of
 * point idx[i] with its own substream (idx[i], iter, Z), so a subset of a
 * full-size pass can be checked at the cost of the subset. */
void orc_gmm_disc_z_subset(const orc_gmm* g, const double* pis, const double* mu, const double* cov,
                           const int* idx, int n_idx, int* z_out, uint64_t seed, uint32_t iter) {
  const int d = g->d, K = g->K;
  double* pmf = (double*)malloc(sizeof(double) * K);
  for (int i = 0; i < n_idx; i++) {
    const int n = idx[i];
    for (int k = 0; k < K; k++) {
      const double* ck = g->shared_cov ? cov : cov + (size_t)k * d * d;
      double prob = 1.0;
      prob *= pis[k];
      prob *= exp(orc_mvnormal_ll(g->Y + (size_t)n * d, mu + (size_t)k * d, ck, d));
      pmf[k] = prob;
    }
    orc_stream s = orc_make(seed, (uint32_t)n, iter, ORC_TAG_Z);
    z_out[i] = orc_unnorm_disc(&s, pmf, K);
  }
  free(pmf);
}

/* Statistics of CgConj.hs:186-246 (AtomicPar over n, sequential here):
 * cnt[k], sum[k] = sum of y, obs[k] = sum of (y - mu[z])(y - mu[z])^T. */
void orc_gmm_stats(const orc_gmm* g, const int* z, const double* mu, int* cnt, double* sum, double* obs) {
  const int d = g->d, K = g->K;
  memset(cnt, 0, sizeof(int) * K);
  if (sum) memset(sum, 0, sizeof(double) * K * d);
  if (obs) memset(obs, 0, sizeof(double) * K * d * d);
  double* diff = (double*)malloc(sizeof(double) * d);
  for (int n = 0; n < g->N; n++) {
    const int k = z[n];
    const double* y = g->Y + (size_t)n * d;
    cnt[k] += 1;
    if (sum) for (int i = 0; i < d; i++) sum[(size_t)k * d + i] += y[i];
    if (obs) {
      for (int i = 0; i < d; i++) diff[i] = y[i] - mu[(size_t)k * d + i];
      double* O = obs + (size_t)k * d * d;
      for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) O[(size_t)i * d + j] += diff[i] * diff[j];
    }
  }
  free(diff);
}

/* ConjGibbs [pis]: Dirichlet(alpha + cnt), element substream (k, iter, PI). */
void orc_gmm_conj_pis(const orc_gmm* g, const int* cnt, double* pis, uint64_t seed, uint32_t iter) {
  orc_dirichlet_vec(g->K, g->alpha, cnt, pis, seed, iter, ORC_TAG_PI);
}

/* ConjGibbs [mu]: per k augur_mvnormal_mvnormal_conj with the covariance of
 * component k (patched argument, CgConj.hs:260-266), substream (k, iter, MU). */
void orc_gmm_conj_mu(const orc_gmm* g, const int* cnt, double* sum, const double* cov, double* mu,
                     uint64_t seed, uint32_t iter) {
  const int d = g->d;
  for (int k = 0; k < g->K; k++) {
    orc_stream s = orc_make(seed, (uint32_t)k, iter, ORC_TAG_MU);
    const double* ck = g->shared_cov ? cov : cov + (size_t)k * d * d;
    orc_mvn_mvn_conj(&s, mu + (size_t)k * d, g->mu0, g->cov0, sum + (size_t)k * d, cnt[k], ck, d);
  }
}

/* ConjGibbs [cov]: augur_invwishart_mvnormal_conj (:751-757): obs += scale0,
 * then InvWishart(cnt + df, obs), substream (k, iter, COV).  obs is updated
 * in place as in the reference. */
void orc_gmm_conj_cov(const orc_gmm* g, const int* cnt, double* obs, double* cov, uint64_t seed,
                      uint32_t iter) {
  const int d = g->d;
  for (int k = 0; k < g->K; k++) {
    double* O = obs + (size_t)k * d * d;
    for (int i = 0; i < d * d; i++) O[i] += g->scale0[i];
    orc_stream s = orc_make(seed, (uint32_t)k, iter, ORC_TAG_COV);
    orc_invwishart_sample(&s, cov + (size_t)k * d * d, cnt[k] + g->df, O, d);
  }
}

/* One augur_step of ConjGibbs [pis] (*) ConjGibbs [mu] (*) ConjGibbs [cov]
 * (*) DiscGibbs [z] (hmvgmm), or ConjGibbs [mu] (*) DiscGibbs [z] (mvgmm;
 * pis and cov fixed). */
void orc_gmm_sweep(const orc_gmm* g, double* pis, double* mu, double* cov, int* z, uint64_t seed,
                   uint32_t iter) {
  const int d = g->d, K = g->K;
  int* cnt = (int*)malloc(sizeof(int) * K);
  double* sum = (double*)malloc(sizeof(double) * K * d);
  double* obs = (double*)malloc(sizeof(double) * K * d * d);
  if (!g->shared_cov) {
    orc_gmm_stats(g, z, mu, cnt, NULL, NULL);
    orc_gmm_conj_pis(g, cnt, pis, seed, iter);
  }
  orc_gmm_stats(g, z, mu, cnt, sum, NULL);
  orc_gmm_conj_mu(g, cnt, sum, cov, mu, seed, iter);
  if (!g->shared_cov) {
    orc_gmm_stats(g, z, mu, cnt, NULL, obs);
    orc_gmm_conj_cov(g, cnt, obs, cov, seed, iter);
  }
  orc_gmm_disc_z(g, pis, mu, cov, z, seed, iter);
  free(cnt); free(sum); free(obs);
}

/* Full conditional of mu[k] (CgLike.hs:236-265 llFnDeclOne): its prior
 * MvNormal(mu0, cov0), then the sum over points of component k. */
double orc_gmm_ll_mu(const orc_gmm* g, const double* muk, int k, const double* cov, const int* z) {
  const int d = g->d;
  const double* ck = g->shared_cov ? cov : cov + (size_t)k * d * d;
  double ll = 0.0;
  ll += orc_mvnormal_ll(muk, g->mu0, g->cov0, d);
  double s = 0.0;
  for (int n = 0; n < g->N; n++)
    if (z[n] == k) s += orc_mvnormal_ll(g->Y + (size_t)n * d, muk, ck, d);
  ll += s;
  return ll;
}

/* ESlice [mu]: augur_mcmc_eslice (augur_mcmclib.h:439-485) per component,
 * substream (k, iter, ESLICE): nu ~ N(mu0, cov0) (d normals), u, theta,
 * then one uniform per shrink.  Returns the number of shrink steps. */
int orc_gmm_eslice(const orc_gmm* g, double* mu, const double* cov, const int* z, uint64_t seed,
                   uint32_t iter) {
  const int d = g->d;
  const double PI2 = 2.0 * 3.14159265358979323846264338327950288;
  double* nu = (double*)malloc(sizeof(double) * d);
  double* prop = (double*)malloc(sizeof(double) * d);
  int shrinks = 0;
  for (int k = 0; k < g->K; k++) {
    double* cur = mu + (size_t)k * d;
    orc_stream s = orc_make(seed, (uint32_t)k, iter, ORC_TAG_ESLICE);
    orc_mvnormal_sample(&s, nu, g->mu0, g->cov0, d);
    double u = orc_uniform(&s);
    double log_y = orc_gmm_ll_mu(g, cur, k, cov, z) + log(u);
    double theta = 0.0 + orc_uniform(&s) * (PI2 - 0.0);
    double tmin = theta - PI2, tmax = theta;
    for (;;) {
      double diff = tmax - tmin;
      if (diff < 1e-8) break;
      for (int i = 0; i < d; i++) {
        double mean_i = g->mu0[i];
        double a = (cur[i] - mean_i) * cos(theta);
        double b = (nu[i] - mean_i) * sin(theta);
        prop[i] = a + b + mean_i;
      }
      double pll = orc_gmm_ll_mu(g, prop, k, cov, z);
      if (pll > log_y) { memcpy(cur, prop, sizeof(double) * d); break; }
      if (theta < 0) tmin = theta; else tmax = theta;
      theta = tmin + orc_uniform(&s) * (tmax - tmin);
      shrinks++;
    }
  }
  free(nu); free(prop);
  return shrinks;
}

/* MWG [mu] ~ MvNormal(mu[k], covp) for k <- 0 until K (CgUserProp.hs:131-260)
 * with the generated correction ll(mu; mu, covp) - ll(mu'; mu, covp) when
 * compat, else 0 (symmetric walk); substream (k, iter, MWG): d normals then
 * the accept uniform.  Returns the number of accepts. */
int orc_gmm_mwg(const orc_gmm* g, double* mu, const double* cov, const int* z, const double* covp,
                int compat, uint64_t seed, uint32_t iter) {
  const int d = g->d;
  double* prop = (double*)malloc(sizeof(double) * d);
  int acc = 0;
  for (int k = 0; k < g->K; k++) {
    double* cur = mu + (size_t)k * d;
    orc_stream s = orc_make(seed, (uint32_t)k, iter, ORC_TAG_MWG);
    orc_mvnormal_sample(&s, prop, cur, covp, d);
    double corr = compat ? orc_mvnormal_ll(cur, cur, covp, d) - orc_mvnormal_ll(prop, cur, covp, d) : 0.0;
    double cl = orc_gmm_ll_mu(g, cur, k, cov, z);
    double pl = orc_gmm_ll_mu(g, prop, k, cov, z);
    double u = orc_uniform(&s);
    if (log(u) < pl - cl + corr) { memcpy(cur, prop, sizeof(double) * d); acc++; }
  }
  free(prop);
  return acc;
}
#undef M_

/* ------------------------------------------------------------------------
 * Scalar conjugate updates over G groups (group g owns observations
 * x[off[g] .. off[g+1])).  Statistics as a generated conj_stat loop would
 * form them (sequential over the observations, CgConj.hs:100-164); draws as
 * cbits/augur_dist.c: beta kinds :185-195 over augur_beta_sample :179-183,
 * gamma kinds :314-336, normal mean :408-412 over augur_normal_sample
 * :404-406.  kind numbering: 0 beta_bernoulli, 1 beta_geometric,
 * 2 gamma_poisson, 3 gamma_exponential, 4 gamma_gammashape,
 * 5 gamma_invgamma, 6 normal_normalmean.  Group g draws from substream
 * (g, iter, ORC_TAG_CONJ).
 * --------------------------------------------------------------------- */
static double orc_beta(orc_stream* s, double a, double b) {
  double x = orc_gamma(s, a, 1.0);
  double y = orc_gamma(s, b, 1.0);
  return x / (x + y);
}

void orc_conj_scalar(int kind, int G, const int* off, const double* x, const double* aux,
                     const double* h0, const double* h1, const double* h2, int per_group,
                     double* stat_sum, double* stat_aux, double* out, uint64_t seed, uint32_t iter) {
  for (int g = 0; g < G; ++g) {
    const int cnt = off[g + 1] - off[g];
    double sum = 0.0, asum = 0.0;
    for (int n = off[g]; n < off[g + 1]; ++n) {
      sum += kind == 5 ? 1.0 / x[n] : x[n];
      if (kind == 4 || kind == 5) asum += aux[n];
    }
    if (stat_sum) stat_sum[g] = sum;
    if (stat_aux) stat_aux[g] = (kind == 4 || kind == 5) ? asum : (double)cnt;
    const int j = per_group ? g : 0;
    const double a = h0[j], b = h1[j];
    orc_stream s = orc_make(seed, (uint32_t)g, iter, ORC_TAG_CONJ);
    double r;
    switch (kind) {
      case 0: r = orc_beta(&s, a + (double)(int)sum, b + (double)(cnt - (int)sum)); break;
      case 1: r = orc_beta(&s, a + (double)cnt, b + (double)(int)sum); break;
      case 2: r = orc_gamma(&s, a + (double)(int)sum, b + (double)cnt); break;
      case 3: r = orc_gamma(&s, a + (double)cnt, b + sum); break;
      case 4:
      case 5: r = orc_gamma(&s, a + asum, b + sum); break;
      default: {
        const double var = h2[j];
        const double pv = 1.0 / (1.0 / b + cnt / var);
        const double pm = (a / b + sum / var) * pv;
        r = pm + sqrt(pv) * orc_normal(&s);
      }
    }
    out[g] = r;
  }
}

/* ---- model log density (ll_mod) and predictive log-likelihoods --------- */

/* augur_dirichlet_ll (augur_dist.c:488-496): no normalising constant. */
static double orc_dirichlet_ll(const double* pt, const double* alpha, int n) {
  double acc = 0.0;
  for (int i = 0; i < n; i++) acc += (alpha[i] - 1.0) * log(pt[i]);
  return acc;
}

/* ll_mod of lda.rv, the function augur_get_curr_ll returns
 * (CgStInit.hs:597-602): the model's factors in model order, each a sum over
 * its comprehension (CgLike.hs:128-147) - augur_dirichlet_ll of the theta
 * rows, of the phi rows, then augur_categorical_ll (log pmf[pt],
 * augur_dist.c:96-102) of every z and every w.  phi is [K][V]. */
double orc_lda_ll_mod(int D, int K, int V, const int* doc_off, const int* w, const int* z,
                      const double* alpha, const double* beta, const double* theta, const double* phi) {
  double ll = 0.0, s = 0.0;
  for (int d = 0; d < D; d++) s += orc_dirichlet_ll(theta + (size_t)d * K, alpha, K);
  ll += s;
  s = 0.0;
  for (int k = 0; k < K; k++) s += orc_dirichlet_ll(phi + (size_t)k * V, beta, V);
  ll += s;
  s = 0.0;
  for (int d = 0; d < D; d++)
    for (int t = doc_off[d]; t < doc_off[d + 1]; t++) s += log(theta[(size_t)d * K + z[t]]);
  ll += s;
  s = 0.0;
  for (int d = 0; d < D; d++)
    for (int t = doc_off[d]; t < doc_off[d + 1]; t++) s += log(phi[(size_t)z[t] * V + w[t]]);
  ll += s;
  return ll;
}

/* augur_multi_lgamma (augur_math.c:80-86), with the reference's log(3.1415). */
static double orc_multi_lgamma(int p, double x) {
  double res = (p * (p - 1) * 0.25) * log(3.1415);
  for (int i = 1; i < p + 1; i++) res += lgamma(x - (i - 1.0) / 2.0);
  return res;
}

#define M_(A, i, j) (A)[(size_t)(i) * d + (j)]

/* augur_invwishart_ll (augur_dist.c:679-711). */
double orc_invwishart_ll(const double* pt, int df, const double* scale, int d) {
  double* L = (double*)malloc(sizeof(double) * d * d);
  double* W = (double*)malloc(sizeof(double) * d * d);
  memcpy(L, scale, sizeof(double) * d * d);
  orc_mat_cholesky(L, d);
  double detPsi = 1.0;
  for (int i = 0; i < d; i++) detPsi *= M_(L, i, i);
  detPsi *= detPsi;
  memcpy(W, pt, sizeof(double) * d * d);
  orc_mat_cholesky(W, d);
  double detX = 1.0;
  for (int i = 0; i < d; i++) detX *= M_(W, i, i);
  detX *= detX;
  orc_mat_cholesky_invert(W, d);
  double tr = 0.0;
  for (int i = 0; i < d; i++) {
    double tmp = 0.0;
    for (int j = 0; j < d; j++) tmp += M_(scale, i, j) * M_(W, j, i);
    tr += tmp;
  }
  double c = -df * d / 2.0 * log(2.0) - orc_multi_lgamma(d, df / 2.0);
  free(L); free(W);
  return c - (df + d + 1.0) / 2.0 * log(detX) + df / 2.0 * log(detPsi) - 0.5 * tr;
}

/* ll_mod of hmvgmm.rv (shared_cov = 0: pis ~ Dirichlet(alpha), mu[k] ~
 * MvNormal(mu0, covs0), cov[k] ~ InvWishart(df, scale0), z[n] ~
 * Categorical(pis), y[n] ~ MvNormal(mu[z[n]], cov[z[n]])) or of mvgmm.rv
 * (shared_cov = 1: mu[k], z[n], y[n] ~ MvNormal(mu[z[n]], covs)), factors in
 * model order as orc_lda_ll_mod. */
double orc_gmm_ll_mod(const orc_gmm* g, const double* pis, const double* mu, const double* cov, const int* z) {
  const int d = g->d, K = g->K;
  double ll = 0.0, s = 0.0;
  if (!g->shared_cov) ll += orc_dirichlet_ll(pis, g->alpha, K);
  for (int k = 0; k < K; k++) s += orc_mvnormal_ll(mu + (size_t)k * d, g->mu0, g->cov0, d);
  ll += s;
  s = 0.0;
  if (!g->shared_cov) {
    for (int k = 0; k < K; k++) s += orc_invwishart_ll(cov + (size_t)k * d * d, g->df, g->scale0, d);
    ll += s;
    s = 0.0;
  }
  for (int n = 0; n < g->N; n++) s += log(pis[z[n]]);
  ll += s;
  s = 0.0;
  for (int n = 0; n < g->N; n++) {
    const double* ck = g->shared_cov ? cov : cov + (size_t)z[n] * d * d;
    s += orc_mvnormal_ll(g->Y + (size_t)n * d, mu + (size_t)z[n] * d, ck, d);
  }
  ll += s;
  return ll;
}

/* log sum_k exp(x_k) as scipy.misc.logsumexp: max + log(sum exp(x - max)). */
static double orc_logsumexp(const double* x, int K) {
  double m = x[0];
  for (int k = 1; k < K; k++) if (x[k] > m) m = x[k];
  if (!(m > -INFINITY)) return m;
  double s = 0.0;
  for (int k = 0; k < K; k++) s += exp(x[k] - m);
  return m + log(s);
}

/* Predictive log-likelihood of held-out tokens for one theta sample
 * (experiments/lda/lda.py:149-173, the inner sum):
 * sum_{d,j} logsumexp_k (log theta[d][k] + log phi[k][w_dj]).  phi [K][V]. */
double orc_lda_pred_ll(int D, int K, int V, const int* doc_off, const int* w, const double* theta,
                       const double* phi) {
  double* tmp = (double*)malloc(sizeof(double) * K);
  double acc = 0.0;
  for (int d = 0; d < D; d++)
    for (int t = doc_off[d]; t < doc_off[d + 1]; t++) {
      for (int k = 0; k < K; k++) tmp[k] = log(theta[(size_t)d * K + k]) + log(phi[(size_t)k * V + w[t]]);
      acc += orc_logsumexp(tmp, K);
    }
  free(tmp);
  return acc;
}

/* Predictive log-likelihood of test points for one (pis, mu, cov) sample
 * (experiments/hmvgmm/hmvgmm.py:143-178, inner_ll):
 * sum_n logsumexp_k (log N(y_n | mu_k, cov_k) + log pis[k]), with the
 * normal log density of augur_mvnormal_ll (the correct one; scipy's logpdf
 * in the experiment).  cov is [K][d][d], or one [d][d] when shared_cov. */
double orc_gmm_pred_ll(int N, int d, int K, int shared_cov, const double* Y, const double* pis,
                       const double* mu, const double* cov) {
  double* tmp = (double*)malloc(sizeof(double) * K);
  double acc = 0.0;
  for (int n = 0; n < N; n++) {
    for (int k = 0; k < K; k++) {
      const double* ck = shared_cov ? cov : cov + (size_t)k * d * d;
      tmp[k] = orc_mvnormal_ll(Y + (size_t)n * d, mu + (size_t)k * d, ck, d) + log(pis[k]);
    }
    acc += orc_logsumexp(tmp, K);
  }
  free(tmp);
  return acc;
}
