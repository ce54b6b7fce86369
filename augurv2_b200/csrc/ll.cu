// Whole-model log densities, held-out predictive log-likelihoods and the
// deterministic variable of dethlr.rv on the device.
//
// * ll_mod: the function the reference's augur_get_curr_ll returns
//   (compiler/augur/src/CudaC/CgStInit.hs:597-602), generated by cgLLMod
//   (compiler/augur/src/Compile/Compile.hs:302-308) as the sum of every
//   factor of the model, each a sum over its comprehension (CgLike.hs:
//   128-147), with the reference's density functions: augur_dirichlet_ll
//   without its normalising constant (cbits/augur_dist.c:488-496),
//   augur_categorical_ll = log pmf[pt] (:96-102), augur_mvnormal_ll
//   (:548-568) and augur_invwishart_ll (:679-711) with augur_multi_lgamma's
//   log(3.1415) (cbits/augur_math.c:80-86).
// * predictive log-likelihood of held-out data for one posterior sample:
//   LDA, sum over held-out tokens of logsumexp_k (log theta[d][k] +
//   log phi[k][w]) (experiments/lda/lda.py:149-173); Gaussian mixtures, sum
//   over test points of logsumexp_k (log N(y | mu_k, cov_k) + log pis[k])
//   (experiments/hmvgmm/hmvgmm.py:143-178).
// * dethlr's bias[n] = sigmoid(dotprod(theta, x[n]) + b)
//   (compiler/augur/test/dethlr.rv; augur_dotprod and augur_expit,
//   cbits/augur_math.c:52-54,119-142) for every chain.
//
// Each reduction is deterministic: the threads of a CTA add in a fixed tree,
// the CTAs' partials are added in CTA order by the last CTA to finish (an
// atomic ticket in the caller's scratch, which returns to zero), and the
// result lands in a device double.  The order differs from the reference's
// sequential loops, so values agree with the CPU oracle to rounding.
#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>

#include "common.cuh"

namespace ab {
namespace {

constexpr int LL_THREADS = 256;
constexpr int LL_MAX_BLOCKS = 148 * 8;
constexpr int LL_MAX_D = 64;

// scratch: ticket (uint32) in the first 256 bytes, then partial f64 [LL_MAX_BLOCKS]
__device__ __forceinline__ bool grid_sum(double v, void* scratch, double* total, double* red) {
  __shared__ int last;
  const double b = block_sum_f64(v, red);
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch);
  double* partial = reinterpret_cast<double*>(static_cast<char*>(scratch) + 256);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = b;
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double s = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(partial + i);
  s = block_sum_f64(s, red);
  if (threadIdx.x == 0) *ticket = 0u;
  *total = s;
  return true;
}

// log N(y | m, cov) with Linv = inverse lower Cholesky factor of cov and
// hdet = log(det cov) / 2, in augur_mvnormal_ll's operation order
// (w = y - m; w' = Linv w row by row; c - hdet - expon / 2).
__device__ __forceinline__ double mvn_ll(const double* y, const double* m, const double* Li, double hdet, int d) {
  const double c = __dmul_rn(__dmul_rn(-0.5, (double)d), log(2.0 * 3.14159265358979323846264338327950288));
  double expon = 0.0;
  for (int i = 0; i < d; ++i) {
    double s = 0.0;
    for (int j = 0; j <= i; ++j) s = __dadd_rn(s, __dmul_rn(Li[(size_t)i * d + j], __dadd_rn(y[j], -m[j])));
    expon = __dadd_rn(expon, __dmul_rn(s, s));
  }
  return __dadd_rn(__dadd_rn(c, -hdet), -__dmul_rn(0.5, expon));
}

// Online log-sum-exp state (max, sum of exp(x - max)), combined across lanes.
struct Lse {
  double m, s;
};
__device__ __forceinline__ void lse_add(Lse& a, double x) {
  if (x > a.m) {
    a.s = a.s * exp(a.m - x) + 1.0;
    a.m = x;
  } else if (x > -INFINITY) {
    a.s += exp(x - a.m);
  }
}
__device__ __forceinline__ Lse lse_merge(Lse a, Lse b) {
  if (b.m > a.m) { Lse t = a; a = b; b = t; }
  if (b.m > -INFINITY) a.s += b.s * exp(b.m - a.m);
  return a;
}
__device__ __forceinline__ double lse_warp(Lse a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Lse b;
    b.m = __shfl_xor_sync(0xffffffffu, a.m, o);
    b.s = __shfl_xor_sync(0xffffffffu, a.s, o);
    a = lse_merge(a, b);
  }
  return a.m > -INFINITY ? a.m + log(a.s) : a.m;
}

// ---- LDA -------------------------------------------------------------------
// mode 0: ll_mod of lda.rv.  mode 1: predictive log-likelihood of the tokens
// (w, doc_off) under theta and phi (z unused).
__global__ void __launch_bounds__(LL_THREADS)
lda_ll_kernel(int mode, int D, int K, int V, int Kp, const int* __restrict__ doc_off, const int* __restrict__ w,
              const int* __restrict__ z, const double* __restrict__ alpha, const double* __restrict__ beta,
              const double* __restrict__ theta, const double* __restrict__ phiT, void* scratch,
              double* __restrict__ out) {
  __shared__ double red[33];
  double v = 0.0;
  const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, gstride = (size_t)gridDim.x * blockDim.x;
  if (mode == 0) {
    for (size_t e = gtid; e < (size_t)D * K; e += gstride)
      v += (alpha[e % K] - 1.0) * log(theta[e]);
    for (size_t e = gtid; e < (size_t)V * K; e += gstride) {
      const size_t vv = e / K, k = e - vv * K;
      v += (beta[vv] - 1.0) * log(phiT[vv * Kp + k]);
    }
    for (int d = blockIdx.x; d < D; d += gridDim.x)
      for (int t = doc_off[d] + threadIdx.x; t < doc_off[d + 1]; t += blockDim.x) {
        const int k = z[t];
        v += log(theta[(size_t)d * K + k]) + log(phiT[(size_t)w[t] * Kp + k]);
      }
  } else {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int d = blockIdx.x; d < D; d += gridDim.x)
      for (int t = doc_off[d] + warp; t < doc_off[d + 1]; t += nw) {
        const double* ph = phiT + (size_t)w[t] * Kp;
        const double* th = theta + (size_t)d * K;
        Lse a{-INFINITY, 0.0};
        for (int k = lane; k < K; k += 32) lse_add(a, log(th[k]) + log(ph[k]));
        const double x = lse_warp(a);
        if (lane == 0) v += x;
      }
  }
  double total;
  if (grid_sum(v, scratch, &total, red) && threadIdx.x == 0) *out = total;
}

// ---- Gaussian mixtures -----------------------------------------------------
struct GmmLL {
  int N, d, K, shared_cov;
  const float* Y;
  const int* z;
  const double* pis;
  const double* mu;
  const double* Linv;     // [Kc][d][d] component tables
  const double* hdet;     // [Kc]
  // ll_mod prior terms
  const double* mu0;
  const double* Linv0;    // [d][d] table of covs0
  const double* hdet0;    // [1]
  const double* alpha;    // [K] (hmvgmm)
  int df;
  const double* scale0;   // [d][d] (hmvgmm)
  const double* hdet_s0;  // [1] log(det scale0) / 2 (hmvgmm)
};

// augur_invwishart_ll (cbits/augur_dist.c:679-711) of cov_k from its tables:
// log det X = 2 hdet_k, X^-1 = Linv_k^T Linv_k, log det Psi = 2 hdet_s0.
__device__ double invwishart_ll_tab(const GmmLL& g, int k) {
  const int d = g.d;
  const double* Li = g.Linv + (size_t)k * d * d;
  double tr = 0.0;
  for (int i = 0; i < d; ++i) {
    double tmp = 0.0;
    for (int j = 0; j < d; ++j) {
      // (X^-1)[j][i] = sum_m Li[m][j] Li[m][i], m >= max(i, j)
      double xji = 0.0;
      for (int m = (i > j ? i : j); m < d; ++m) xji += Li[(size_t)m * d + j] * Li[(size_t)m * d + i];
      tmp += g.scale0[(size_t)i * d + j] * xji;
    }
    tr += tmp;
  }
  double mlg = (d * (d - 1) * 0.25) * log(3.1415);
  for (int i = 1; i < d + 1; ++i) mlg += lgamma(g.df / 2.0 - (i - 1.0) / 2.0);
  const double c = -g.df * d / 2.0 * log(2.0) - mlg;
  const double log_detX = 2.0 * g.hdet[k], log_detPsi = 2.0 * *g.hdet_s0;
  return c - (g.df + d + 1.0) / 2.0 * log_detX + g.df / 2.0 * log_detPsi - 0.5 * tr;
}

// mode 0: ll_mod of hmvgmm.rv (shared_cov 0) or mvgmm.rv (shared_cov 1);
// mode 1: predictive log-likelihood of the points Y.
__global__ void __launch_bounds__(LL_THREADS)
gmm_ll_kernel(int mode, GmmLL g, void* scratch, double* __restrict__ out) {
  __shared__ double red[33];
  const int d = g.d;
  double y[LL_MAX_D];
  double v = 0.0;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += gridDim.x * blockDim.x) {
    for (int i = 0; i < d; ++i) y[i] = (double)g.Y[(size_t)n * d + i];
    if (mode == 0) {
      const int k = g.z[n], kc = g.shared_cov ? 0 : k;
      v += log(g.pis[k]) + mvn_ll(y, g.mu + (size_t)k * d, g.Linv + (size_t)kc * d * d, g.hdet[kc], d);
    } else {
      Lse a{-INFINITY, 0.0};
      for (int k = 0; k < g.K; ++k) {
        const int kc = g.shared_cov ? 0 : k;
        lse_add(a, mvn_ll(y, g.mu + (size_t)k * d, g.Linv + (size_t)kc * d * d, g.hdet[kc], d) + log(g.pis[k]));
      }
      v += a.m > -INFINITY ? a.m + log(a.s) : a.m;
    }
  }
  double total;
  if (!grid_sum(v, scratch, &total, red)) return;
  if (mode == 1) {
    if (threadIdx.x == 0) *out = total;
    return;
  }
  // the parameters' own factors, by the last CTA
  __shared__ double pri[3];
  if (threadIdx.x < 3) pri[threadIdx.x] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    if (!g.shared_cov)
      for (int k = 0; k < g.K; ++k) s += (g.alpha[k] - 1.0) * log(g.pis[k]);
    pri[0] = s;
  }
  double mv = 0.0, iw = 0.0;
  for (int k = threadIdx.x; k < g.K; k += blockDim.x) {
    mv += mvn_ll(g.mu + (size_t)k * d, g.mu0, g.Linv0, *g.hdet0, d);
    if (!g.shared_cov) iw += invwishart_ll_tab(g, k);
  }
  mv = block_sum_f64(mv, red);
  iw = block_sum_f64(iw, red);
  if (threadIdx.x == 0) *out = pri[0] + mv + iw + total;
}

// ---- dethlr's deterministic bias -------------------------------------------
__global__ void __launch_bounds__(LL_THREADS)
hlr_det_kernel(int N, int D, int ldx, int x_dtype, const void* __restrict__ X, int C, int has_b,
               const double* __restrict__ pars, double* __restrict__ out) {
  const size_t total = (size_t)C * N;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e / N), n = (int)(e - (size_t)c * N);
    const double* th = pars + (size_t)c * (D + 2);
    double t = 0.0;
    for (int j = 0; j < D; ++j) {
      const double x = x_dtype == AB_BF16
                           ? (double)__bfloat162float(static_cast<const __nv_bfloat16*>(X)[(size_t)n * ldx + j])
                           : (double)static_cast<const float*>(X)[(size_t)n * ldx + j];
      t = __dadd_rn(t, __dmul_rn(th[j], x));
    }
    if (has_b) t = __dadd_rn(t, th[D]);
    out[e] = 1.0 / (1.0 + exp(-t));
  }
}

int grid_for(size_t items) {
  size_t b = (items + LL_THREADS - 1) / LL_THREADS;
  if (b < 1) b = 1;
  return (int)(b < (size_t)LL_MAX_BLOCKS ? b : (size_t)LL_MAX_BLOCKS);
}

}  // namespace
}  // namespace ab

using namespace ab;

extern "C" size_t ab_ll_scratch_bytes(void) { return 256 + sizeof(double) * LL_MAX_BLOCKS; }

static int lda_ll_common(int mode, int D, int K, int V, const int* doc_off, const int* w, const int* z,
                         const double* alpha, const double* beta, const double* theta, const double* phiT,
                         double* out, void* scratch, void* stream) {
  AB_REQUIRE(D > 0 && K > 0 && V > 0, AB_ERR_ARG, "lda ll: sizes must be positive (D=%d K=%d V=%d)", D, K, V);
  AB_REQUIRE(doc_off && w && theta && phiT && out && scratch, AB_ERR_ARG, "lda ll: null pointer");
  AB_REQUIRE(mode == 1 || (z && alpha && beta), AB_ERR_ARG, "ab_lda_ll_mod: null pointer");
  const int Kp = ab_lda_phi_stride(K);
  const int nb = grid_for(mode == 0 ? std::max((size_t)D * K, (size_t)V * K) : (size_t)D * 32);
  lda_ll_kernel<<<nb, LL_THREADS, 0, as_stream(stream)>>>(mode, D, K, V, Kp, doc_off, w, z, alpha, beta, theta,
                                                          phiT, scratch, out);
  AB_LAUNCH_CHECK("lda_ll_kernel");
  return AB_OK;
}

extern "C" int ab_lda_ll_mod(int D, int K, int V, const int* doc_off, const int* w, const int* z,
                             const double* alpha, const double* beta, const double* theta, const double* phiT,
                             double* out, void* scratch, void* stream) {
  return lda_ll_common(0, D, K, V, doc_off, w, z, alpha, beta, theta, phiT, out, scratch, stream);
}

extern "C" int ab_lda_pred_ll(int D, int K, int V, const int* doc_off, const int* w, const double* theta,
                              const double* phiT, double* out, void* scratch, void* stream) {
  return lda_ll_common(1, D, K, V, doc_off, w, nullptr, nullptr, nullptr, theta, phiT, out, scratch, stream);
}

static int gmm_ll_common(int mode, const GmmLL& g, double* out, void* scratch, void* stream) {
  AB_REQUIRE(g.N > 0 && g.d > 0 && g.d <= LL_MAX_D && g.K > 0, AB_ERR_ARG,
             "gmm ll: need N > 0, 0 < d <= %d, K > 0 (N=%d d=%d K=%d)", LL_MAX_D, g.N, g.d, g.K);
  AB_REQUIRE(g.Y && g.pis && g.mu && g.Linv && g.hdet && out && scratch, AB_ERR_ARG, "gmm ll: null pointer");
  gmm_ll_kernel<<<grid_for((size_t)g.N), LL_THREADS, 0, as_stream(stream)>>>(mode, g, scratch, out);
  AB_LAUNCH_CHECK("gmm_ll_kernel");
  return AB_OK;
}

extern "C" int ab_gmm_ll_mod(int N, int d, int K, int shared_cov, const float* Y, const int* z, const double* pis,
                             const double* mu, const double* Linv, const double* hdet, const double* mu0,
                             const double* Linv0, const double* hdet0, const double* alpha, int df,
                             const double* scale0, const double* hdet_s0, double* out, void* scratch,
                             void* stream) {
  AB_REQUIRE(z && mu0 && Linv0 && hdet0, AB_ERR_ARG, "ab_gmm_ll_mod: null pointer");
  AB_REQUIRE(shared_cov || (alpha && scale0 && hdet_s0 && df > d - 1), AB_ERR_ARG,
             "ab_gmm_ll_mod: hmvgmm needs alpha, scale0, hdet_s0 and df > d - 1");
  GmmLL g{N, d, K, shared_cov, Y, z, pis, mu, Linv, hdet, mu0, Linv0, hdet0, alpha, df, scale0, hdet_s0};
  return gmm_ll_common(0, g, out, scratch, stream);
}

extern "C" int ab_gmm_pred_ll(int N, int d, int K, int shared_cov, const float* Y, const double* pis,
                              const double* mu, const double* Linv, const double* hdet, double* out, void* scratch,
                              void* stream) {
  GmmLL g{N, d, K, shared_cov, Y, nullptr, pis, mu, Linv, hdet, nullptr, nullptr, nullptr, nullptr, 0, nullptr,
          nullptr};
  return gmm_ll_common(1, g, out, scratch, stream);
}

extern "C" int ab_hlr_det(const ab_hlr_model* m, int C, const double* pars, double* out, void* stream) {
  AB_REQUIRE(m && pars && out && m->X, AB_ERR_ARG, "ab_hlr_det: null pointer");
  AB_REQUIRE(m->N > 0 && m->D > 0 && C > 0 && m->ldx >= m->D, AB_ERR_ARG, "ab_hlr_det: bad sizes");
  AB_REQUIRE(m->x_dtype == AB_F32 || m->x_dtype == AB_BF16, AB_ERR_ARG, "ab_hlr_det: X must be f32 or bf16");
  hlr_det_kernel<<<grid_for((size_t)C * m->N), LL_THREADS, 0, as_stream(stream)>>>(
      m->N, m->D, m->ldx, m->x_dtype, m->X, C, m->has_b, pars, out);
  AB_LAUNCH_CHECK("hlr_det_kernel");
  return AB_OK;
}
