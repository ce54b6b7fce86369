// Batched HMC driver: C chains advance together, one thread block per chain
// for the vector updates, with the log density and gradient supplied by the
// caller between the steps (the tensor-core HLR pass, or a gradient
// surrogate for the trajectory with the exact log density at its end).
//
// One iteration, following h_augur_mcmc_hmc / h_augur_mcmc_leapfrog
// (cbits/augur_mcmclib.h:343-424) for each chain:
//   begin   p ~ N(0, I); eps_c = eps0 (1 + jitter (2u - 1)); H0 = -logp + |p|^2/2;
//           save theta0, g0, logp0; p += eps/2 g; theta += eps p
//   step    (L - 1 times, after a gradient g at theta)  p += eps g; theta += eps p
//   final   (after logp_new, g_new at the end point)    p += eps/2 g_new;
//           H1 = -logp_new + |p|^2/2; accept iff log u < H0 - H1 (FP64),
//           else restore theta0, g0, logp0.
// The step count is the caller's; the reference draws it from a jittered
// simulation length, here every chain takes the same L and the step size is
// jittered per chain.  Energies and the accept test are FP64; positions,
// momenta and gradients FP32.  Randomness: Philox streams keyed by
// (seed, chain, iteration) with tags MOM (momenta, one normal per
// coordinate) and HMC (jitter at position 0, accept uniform at position 1).
// The iteration counter lives on the device and is advanced by final, so a
// captured CUDA graph of one iteration replays correctly.
#include <math.h>

#include "common.cuh"
#include "philox.cuh"

namespace ab {
namespace {

__global__ void __launch_bounds__(256) hmcb_begin_kernel(ab_hmcb_state s) {
  __shared__ double red[33];
  __shared__ float eps_sh;
  const int c = blockIdx.x, D = s.D;
  const uint32_t it = (uint32_t)*s.iter;
  if (threadIdx.x == 0) {
    Stream h = make_stream(s.seed, (uint32_t)c, it, TAG_HMC);
    const double u = h.uniform();
    const float e = (float)((double)*s.eps0 * (1.0 + (double)s.jitter * (2.0 * u - 1.0)));
    eps_sh = e;
    s.eps_c[c] = e;
    s.logp0[c] = s.logp_cur[c];
  }
  __syncthreads();
  const float eps = eps_sh;
  double k = 0.0;
  const size_t off = (size_t)c * D;
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    Stream m = make_stream(s.seed, (uint32_t)c, it, TAG_MOM);
    m.pos = (uint32_t)d;
    float p = (float)m.normal();
    k += 0.5 * (double)p * (double)p;
    const float th = s.theta[off + d], g = s.g_cur[off + d];
    s.theta0[off + d] = th;
    s.g0[off + d] = g;
    p += 0.5f * eps * g;
    s.p[off + d] = p;
    s.theta[off + d] = th + eps * p;
  }
  k = block_sum_f64(k, red);
  if (threadIdx.x == 0) s.H0[c] = -s.logp_cur[c] + k;
}

__global__ void __launch_bounds__(256) hmcb_step_kernel(ab_hmcb_state s, const float* __restrict__ g) {
  const int c = blockIdx.x, D = s.D;
  const float eps = s.eps_c[c];
  const size_t off = (size_t)c * D;
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    const float p = s.p[off + d] + eps * g[off + d];
    s.p[off + d] = p;
    s.theta[off + d] += eps * p;
  }
}

__global__ void __launch_bounds__(256) hmcb_final_kernel(ab_hmcb_state s, const float* __restrict__ g_new,
                                                         const double* __restrict__ logp_new) {
  __shared__ double red[33];
  __shared__ int acc_sh;
  const int c = blockIdx.x, D = s.D;
  const float eps = s.eps_c[c];
  const size_t off = (size_t)c * D;
  double k = 0.0;
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    const float p = s.p[off + d] + 0.5f * eps * g_new[off + d];
    s.p[off + d] = p;
    k += 0.5 * (double)p * (double)p;
  }
  k = block_sum_f64(k, red);
  if (threadIdx.x == 0) {
    const uint32_t it = (uint32_t)*s.iter;
    Stream h = make_stream(s.seed, (uint32_t)c, it, TAG_HMC);
    h.pos = 1;
    const double u = h.uniform();
    const double H1 = -logp_new[c] + k;
    const double dH = s.H0[c] - H1;
    const bool ok = isfinite(H1) && log(u) < dH;
    acc_sh = ok;
    double* st = s.stats + (size_t)AB_HMCB_STATS * c;
    st[0] += ok ? 1.0 : 0.0;
    st[1] += isfinite(dH) ? (dH >= 0.0 ? 1.0 : exp(dH)) : 0.0;
    // energy error above the divergence bound, or not finite
    st[2] += (dH > -AB_DIVERGENCE_DH) ? 0.0 : 1.0;
    s.logp_cur[c] = ok ? logp_new[c] : s.logp0[c];
  }
  __syncthreads();
  const bool ok = acc_sh;
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    if (ok) {
      s.g_cur[off + d] = g_new[off + d];
    } else {
      s.theta[off + d] = s.theta0[off + d];
      s.g_cur[off + d] = s.g0[off + d];
    }
  }
}

// Advances the device iteration counter after every chain's final step.
__global__ void hmcb_advance_kernel(long long* iter) { *iter += 1; }

int check_state(const ab_hmcb_state* s) {
  AB_REQUIRE(s, AB_ERR_ARG, "hmcb: null state");
  AB_REQUIRE(s->C > 0 && s->C <= 1 << 20 && s->D > 0, AB_ERR_ARG, "hmcb: bad sizes C=%d D=%d", s->C, s->D);
  AB_REQUIRE(s->iter && s->eps0 && s->theta && s->p && s->g_cur && s->logp_cur && s->theta0 && s->g0 &&
                 s->logp0 && s->H0 && s->eps_c && s->stats,
             AB_ERR_ARG, "hmcb: null state pointer");
  AB_REQUIRE(s->jitter >= 0.0f && s->jitter < 1.0f, AB_ERR_ARG, "hmcb: jitter must be in [0, 1)");
  return AB_OK;
}

}  // namespace
}  // namespace ab

using namespace ab;

extern "C" int ab_hmcb_begin(const ab_hmcb_state* s, void* stream) {
  int rc = check_state(s);
  if (rc) return rc;
  hmcb_begin_kernel<<<s->C, 256, 0, as_stream(stream)>>>(*s);
  AB_LAUNCH_CHECK("hmcb_begin_kernel");
  return AB_OK;
}

extern "C" int ab_hmcb_step(const ab_hmcb_state* s, const float* g, void* stream) {
  int rc = check_state(s);
  if (rc) return rc;
  AB_REQUIRE(g, AB_ERR_ARG, "ab_hmcb_step: null gradient");
  hmcb_step_kernel<<<s->C, 256, 0, as_stream(stream)>>>(*s, g);
  AB_LAUNCH_CHECK("hmcb_step_kernel");
  return AB_OK;
}

extern "C" int ab_hmcb_final(const ab_hmcb_state* s, const float* g_new, const double* logp_new, void* stream) {
  int rc = check_state(s);
  if (rc) return rc;
  AB_REQUIRE(g_new && logp_new, AB_ERR_ARG, "ab_hmcb_final: null pointer");
  hmcb_final_kernel<<<s->C, 256, 0, as_stream(stream)>>>(*s, g_new, logp_new);
  AB_LAUNCH_CHECK("hmcb_final_kernel");
  hmcb_advance_kernel<<<1, 1, 0, as_stream(stream)>>>(s->iter);
  AB_LAUNCH_CHECK("hmcb_advance_kernel");
  return AB_OK;
}
