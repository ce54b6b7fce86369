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
