// Scalar conjugate updates: the seven one-parameter conjugate pairs of the
// reference distribution library (cbits/augur_dist.c:185-195, 314-336,
// 408-412) as one batched Gibbs step over G groups.
//
// Data layout: the observations of group g are x[off[g] .. off[g+1]) (the
// flattening of a ragged Vec (Vec Real), like the LDA documents); `aux`
// holds a per-observation known shape for the two kinds whose likelihood
// has one.  One warp per group forms the sufficient statistics (lanes
// stride over the group's observations, a fixed xor tree adds the lane
// partials: deterministic, equal to the reference's sequential sum up to
// rounding, exact for integer-valued data) and lane 0 draws the group's
// parameter from its conjugate posterior on Philox substream
// (g, iter, TAG_CONJ), consuming the uniforms in the order of the
// reference sampler.
#include <cmath>

#include "common.cuh"
#include "dist.cuh"

namespace ab {

constexpr int CONJ_THREADS = 256;

struct ConjHyp {
  const double* h0;
  const double* h1;
  const double* h2;
  int per_group;
  __device__ __forceinline__ double get(const double* h, int g) const { return h[per_group ? g : 0]; }
};

// Posterior parameters outside the sampler's domain (non-positive or NaN
// shapes, rates or variances) give NaN instead of entering the rejection
// loop.
__device__ __forceinline__ bool pos_finite(double v) { return v > 0.0 && v < INFINITY; }

// augur_beta_sample (augur_dist.c:179-183): x / (x + y) with
// x ~ Gamma(a, 1) drawn before y ~ Gamma(b, 1).
__device__ __forceinline__ double beta_draw(Stream& s, double a, double b) {
  if (!pos_finite(a) || !pos_finite(b)) return NAN;
  const double x = gamma_draw(s, a, 1.0);
  const double y = gamma_draw(s, b, 1.0);
  return x / __dadd_rn(x, y);
}

__device__ __forceinline__ double gamma_post(Stream& s, double shape, double rate) {
  if (!pos_finite(shape) || !pos_finite(rate)) return NAN;
  return gamma_draw(s, shape, rate);
}

__global__ void __launch_bounds__(CONJ_THREADS)
conj_scalar_kernel(int kind, int G, const int* __restrict__ off, const double* __restrict__ x,
                   const double* __restrict__ aux, ConjHyp hyp, double* __restrict__ stat_sum,
                   double* __restrict__ stat_aux, double* __restrict__ out, uint64_t seed, uint32_t iter) {
  const int lane = threadIdx.x & 31;
  const int g = blockIdx.x * (CONJ_THREADS / 32) + (threadIdx.x >> 5);
  if (g >= G) return;
  const int lo = off[g], hi = off[g + 1];
  double s = 0.0, a = 0.0;
  for (int n = lo + lane; n < hi; n += 32) {
    const double v = x[n];
    // gamma_invgamma takes the sum of reciprocals of the observations
    s = __dadd_rn(s, kind == AB_CONJ_GAMMA_INVGAMMA ? 1.0 / v : v);
    if (aux) a = __dadd_rn(a, aux[n]);
  }
  s = warp_sum_f64(s);
  a = warp_sum_f64(a);
  if (lane) return;
  const int cnt = hi - lo;
  if (stat_sum) stat_sum[g] = s;
  if (stat_aux) stat_aux[g] = aux ? a : (double)cnt;
  Stream st = make_stream(seed, (uint32_t)g, iter, TAG_CONJ);
  const double h0 = hyp.get(hyp.h0, g), h1 = hyp.get(hyp.h1, g);
  double r;
  switch (kind) {
    case AB_CONJ_BETA_BERNOULLI: {   // augur_dist.c:185-189
      const int sum = (int)s;
      r = beta_draw(st, __dadd_rn(h0, (double)sum), __dadd_rn(h1, (double)(cnt - sum)));
      break;
    }
    case AB_CONJ_BETA_GEOMETRIC: {   // :191-195
      const int sum = (int)s;
      r = beta_draw(st, __dadd_rn(h0, (double)cnt), __dadd_rn(h1, (double)sum));
      break;
    }
    case AB_CONJ_GAMMA_POISSON: {    // :314-318
      const int sum = (int)s;
      r = gamma_post(st, __dadd_rn(h0, (double)sum), __dadd_rn(h1, (double)cnt));
      break;
    }
    case AB_CONJ_GAMMA_EXPONENTIAL:  // :320-324
      r = gamma_post(st, __dadd_rn(h0, (double)cnt), __dadd_rn(h1, s));
      break;
    case AB_CONJ_GAMMA_GAMMASHAPE:   // :326-330
    case AB_CONJ_GAMMA_INVGAMMA:     // :332-336
      r = gamma_post(st, __dadd_rn(h0, a), __dadd_rn(h1, s));
      break;
    default: {                       // AB_CONJ_NORMAL_NORMALMEAN, :408-412
      const double var = hyp.get(hyp.h2, g);
      if (!pos_finite(h1) || !pos_finite(var)) { r = NAN; break; }
      const double pv = 1.0 / __dadd_rn(1.0 / h1, (double)cnt / var);
      const double pm = __dmul_rn(__dadd_rn(h0 / h1, s / var), pv);
      // augur_normal_sample (augur_dist.c:404-406)
      r = __dadd_rn(pm, __dmul_rn(sqrt(pv), st.normal()));
      break;
    }
  }
  out[g] = r;
}

}  // namespace ab

using namespace ab;

extern "C" int ab_conj_scalar(int kind, int G, const int* off, const double* x, const double* aux,
                              const double* h0, const double* h1, const double* h2, int per_group,
                              double* stat_sum, double* stat_aux, double* out, uint64_t seed,
                              uint32_t iter, void* stream) {
  AB_REQUIRE(kind >= AB_CONJ_BETA_BERNOULLI && kind <= AB_CONJ_NORMAL_NORMALMEAN, AB_ERR_ARG,
             "conj kind %d out of range", kind);
  AB_REQUIRE(G >= 0, AB_ERR_ARG, "G must be >= 0");
  if (G == 0) return AB_OK;
  AB_REQUIRE(off && out && h0 && h1, AB_ERR_ARG, "off, out, h0 and h1 are required");
  AB_REQUIRE(kind != AB_CONJ_NORMAL_NORMALMEAN || h2, AB_ERR_ARG,
             "normal_normalmean needs h2 (the observation variance)");
  const bool shaped = kind == AB_CONJ_GAMMA_GAMMASHAPE || kind == AB_CONJ_GAMMA_INVGAMMA;
  AB_REQUIRE(!shaped || aux, AB_ERR_ARG, "this kind needs aux (the observations' known shapes)");
  AB_REQUIRE(per_group == 0 || per_group == 1, AB_ERR_ARG, "per_group must be 0 or 1");
  ConjHyp hyp{h0, h1, h2, per_group};
  const int blocks = (int)(((long long)G + CONJ_THREADS / 32 - 1) / (CONJ_THREADS / 32));
  conj_scalar_kernel<<<blocks, CONJ_THREADS, 0, as_stream(stream)>>>(
      kind, G, off, x, shaped ? aux : nullptr, hyp, stat_sum, stat_aux, out, seed, iter);
  AB_LAUNCH_CHECK("conj_scalar_kernel");
  return AB_OK;
}
