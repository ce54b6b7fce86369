// Device samplers shared by the Gibbs and HMC kernels.  Each follows the
// reference distribution library (cbits/augur_dist.c) operation for
// operation in binary64, drawing from a Philox substream (philox.cuh).
#pragma once
#include "philox.cuh"

namespace ab {

// Marsaglia & Tsang (2000) for shape >= 1 (cbits/augur_dist.c:287-300).
// The binary64 mul/add steps are spelled with _rn intrinsics so that no
// multiply-add is contracted, as in the reference's libcpu build.
__device__ __forceinline__ double gamma_ge1(Stream& s, double alpha) {
  const double d = __dadd_rn(alpha, -1.0 / 3.0);
  const double c = 1.0 / sqrt(__dmul_rn(9.0, d));
  const double neg_inv_c = -1.0 / c;
  for (int tries = 0; tries < 1000000; ++tries) {
    double z = s.normal();
    double u = s.uniform();
    double t = __dadd_rn(1.0, __dmul_rn(c, z));
    double V = __dmul_rn(__dmul_rn(t, t), t);
    if (z > neg_inv_c) {
      // Marsaglia & Tsang's squeeze: u < 1 - 0.0331 z^4 lies inside the
      // acceptance region log(u) < rhs for every d >= 1/3 (here d >= 2/3;
      // near z = 0, rhs ~ -z^4 / (108 d) against -0.0331 z^4), so the draw
      // is the reference's without its two logarithms.  The two tests can
      // only disagree where the binary64 rounding of rhs (~1e-16 d) exceeds
      // the bound's margin, i.e. for u within ~1e-16 d of the squeeze
      // boundary at |z| < ~1e-3: an event of probability below 1e-16 per draw
      // for the shapes of these samplers.
      const double z2 = __dmul_rn(z, z);
      if (u < __dadd_rn(1.0, -__dmul_rn(0.0331, __dmul_rn(z2, z2)))) return __dmul_rn(d, V);
      double rhs = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(0.5, z), z), d),
                                       -__dmul_rn(d, V)),
                             __dmul_rn(d, log(V)));
      if (log(u) < rhs) return __dmul_rn(d, V);
    }
  }
  return __dmul_rn(d, 1.0);  // unreachable in practice (acceptance > 95%)
}

// cbits/augur_dist.c:302-312: boost shape < 1 through Gamma(shape + 1).
// The rejection loop is written once for both cases (its shape argument
// selected first), so that a warp whose lanes mix shapes below and above 1
// runs one copy of the loop instead of the two branches' copies in turn;
// every lane still performs the reference's operations in its order.
__device__ __forceinline__ double gamma_draw(Stream& s, double shape, double rate) {
  const double scale = 1.0 / rate;
  const bool boost = shape < 1.0;
  double x = gamma_ge1(s, boost ? __dadd_rn(shape, 1.0) : shape);
  if (boost) {
    double u = s.uniform();
    x = __dmul_rn(x, pow(u, 1.0 / shape));
  }
  return __dmul_rn(x, scale);
}

}  // namespace ab
