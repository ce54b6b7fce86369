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

// The first try of gamma_draw's Marsaglia-Tsang loop and, for a boosted
// shape, its boost (substream positions 0, 1 and 2), decided by the squeeze
// alone.  Returns true with the draw gamma_draw would return when that try
// accepts by the squeeze (about 95% of draws at the shapes of the Gibbs
// samplers); returns false otherwise - a rejected try, or one that needs the
// logarithmic test - with the try's normal and uniform in z_out, u_out, from
// which gamma_draw_resume completes the draw in a later pass.  Straight-line
// code: no lane of a warp waits on another lane's rejection loop.
__device__ __forceinline__ bool gamma_first_try(Stream& s, double shape, double rate, double& out,
                                                double& z_out, double& u_out) {
  const bool boost = shape < 1.0;
  const double a = boost ? __dadd_rn(shape, 1.0) : shape;
  const double d = __dadd_rn(a, -1.0 / 3.0);
  const double c = 1.0 / sqrt(__dmul_rn(9.0, d));
  const double z = s.normal();
  const double u = s.uniform();
  const double t = __dadd_rn(1.0, __dmul_rn(c, z));
  const double V = __dmul_rn(__dmul_rn(t, t), t);
  const double z2 = __dmul_rn(z, z);
  z_out = z;
  u_out = u;
  if (!(z > -1.0 / c) || !(u < __dadd_rn(1.0, -__dmul_rn(0.0331, __dmul_rn(z2, z2))))) return false;
  double x = __dmul_rn(d, V);
  if (boost) {
    const double ub = s.uniform();
    x = __dmul_rn(x, pow(ub, 1.0 / shape));
  }
  out = __dmul_rn(x, 1.0 / rate);
  return true;
}

// Completes a draw gamma_first_try left undecided, from that first try's
// normal z1 and uniform u1 and the stream positioned after them (position 2):
// the first try's logarithmic test (when z1 passed the support test), then
// gamma_ge1's further tries, then the boost.  The same operations in the same
// order as gamma_draw from position 0, so the same value.
__device__ __forceinline__ double gamma_draw_resume(Stream& s, double shape, double rate, double z1, double u1) {
  const double scale = 1.0 / rate;
  const bool boost = shape < 1.0;
  const double a = boost ? __dadd_rn(shape, 1.0) : shape;
  const double d = __dadd_rn(a, -1.0 / 3.0);
  const double c = 1.0 / sqrt(__dmul_rn(9.0, d));
  const double neg_inv_c = -1.0 / c;
  double x = 0.0;
  bool done = false;
  if (z1 > neg_inv_c) {
    const double t = __dadd_rn(1.0, __dmul_rn(c, z1));
    const double V = __dmul_rn(__dmul_rn(t, t), t);
    const double rhs = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(0.5, z1), z1), d), -__dmul_rn(d, V)),
                                 __dmul_rn(d, log(V)));
    if (log(u1) < rhs) {
      x = __dmul_rn(d, V);
      done = true;
    }
  }
  if (!done) x = gamma_ge1(s, a);
  if (boost) {
    const double u = s.uniform();
    x = __dmul_rn(x, pow(u, 1.0 / shape));
  }
  return __dmul_rn(x, scale);
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
