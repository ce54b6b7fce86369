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
