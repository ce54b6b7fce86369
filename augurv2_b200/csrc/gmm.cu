// Gaussian mixtures: the DiscGibbs assignment draw, the conjugate statistics
// and draws of ConjGibbs [pis] / [mu] / [cov], and the ESlice / MWG moves of
// the component means, for the models compiler/augur/test/mvgmm.rv (shared
// covariance, fixed weights) and hmvgmm.rv (weights ~ Dirichlet, covariances
// ~ InvWishart).
//
// Layout in HBM: Y f32 [N][d] (data), z int32 [N], pis f64 [K],
// mu f64 [K][d], cov f64 [Kc][d][d] (Kc = 1 when shared), all row-major;
// Linv f64 [Kc][d][d] and hdet f64 [Kc] are per-sweep derived tables.
//
// Arithmetic is binary64 without contraction (this file is compiled with
// -fmad=false and uses _rn intrinsics).  The reference's d x d routines
// (cbits/augur_matop.c:312-420) are in-place sequential loops; the warp
// routines below compute every element with the same operand order, reading
// the values the in-place reference would read at that point, so their
// results are bit-identical; only the order in which independent elements
// are produced changes.  The per-point log-density uses the Cholesky inverse
// of the component covariance computed once per sweep — the same binary64
// values the reference recomputes for every (point, component).
#include "common.cuh"
#include "dist.cuh"

namespace ab {

constexpr int GMM_MAX_D = 64;
constexpr int GMM_MAX_K = 64;
constexpr int GMM_THREADS = 256;
constexpr int GMM_STAT_CTAS = 296;

#define GM(A, i, j) (A)[(size_t)(i) * d + (j)]

// ---- warp-level matrix routines (one full warp, matrices in shared memory)

// augur_mat_cholesky (:312-328), column by column; (i, j) uses row i and
// row j left of j, and the diagonal (j, j) - all final before column j.
__device__ void w_chol(double* A, int d) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < d; ++j) {
    if (lane == 0) {
      double s = 0.0;
      for (int k = 0; k < j; ++k) s = __dadd_rn(s, __dmul_rn(GM(A, j, k), GM(A, j, k)));
      GM(A, j, j) = __dsqrt_rn(__dadd_rn(GM(A, j, j), -s));
    }
    __syncwarp();
    for (int i = j + 1 + lane; i < d; i += 32) {
      double s = 0.0;
      for (int k = 0; k < j; ++k) s = __dadd_rn(s, __dmul_rn(GM(A, i, k), GM(A, j, k)));
      GM(A, i, j) = __dmul_rn(__ddiv_rn(1.0, GM(A, j, j)), __dadd_rn(GM(A, i, j), -s));
    }
    __syncwarp();
  }
}

// augur_mat_lower_trmi (:335-345).  In the in-place loop the entries above
// the diagonal of column c come out as exact zeros before any lower entry of
// the column is formed, so each column is an independent forward
// substitution over the original factor; the zero terms it skips change
// nothing.  One lane per column; T receives the original factor, which the
// sequential loop would still see in the columns not yet processed.
__device__ void w_trmi(double* L, double* T, int d) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < d * d; e += 32) T[e] = L[e];
  __syncwarp();
  for (int c = lane; c < d; c += 32) {
    for (int m = c; m < d; ++m) {
      double b = (c == m) ? 1.0 : 0.0;
      for (int i = c; i < m; ++i) b = __dadd_rn(b, -__dmul_rn(GM(T, m, i), GM(L, i, c)));
      GM(L, m, c) = __ddiv_rn(b, GM(T, m, m));
    }
  }
  __syncwarp();
  for (int e = lane; e < d * d; e += 32) {
    const int r = e / d, c = e - r * d;
    if (r < c) L[e] = 0.0;
  }
  __syncwarp();
}

// augur_mat_cholesky_invert (:363-375): trmi, then for each column c and row
// r >= c (in order) A[r][c] = sum_{k=c}^{d-1} A[k][r] A[k][c] with the
// column's earlier rows already replaced, then the lower part mirrored.
// Columns only read their own progress and later columns, which the
// reference has not yet touched, so they run in parallel from a copy T.
__device__ void w_cholinv(double* A, double* T, int d) {
  const int lane = threadIdx.x & 31;
  w_trmi(A, T, d);
  for (int e = lane; e < d * d; e += 32) T[e] = A[e];
  __syncwarp();
  for (int c = lane; c < d; c += 32) {
    for (int r = c; r < d; ++r) {
      double acc = 0.0;
      for (int k = c; k < d; ++k) {
        const double akc = (k < r) ? GM(A, k, c) : GM(T, k, c);
        acc = __dadd_rn(acc, __dmul_rn(GM(T, k, r), akc));
      }
      GM(A, r, c) = acc;
    }
  }
  __syncwarp();
  for (int e = lane; e < d * d; e += 32) {
    const int r = e / d, c = e - r * d;
    if (r < c) A[e] = GM(A, c, r);
  }
  __syncwarp();
}

// augur_mat_trvm (:398-406): v = L v (row i uses the original v[0..i]).
__device__ void w_trvm(const double* L, double* v, double* tmp, int d) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < d; i += 32) {
    double s = 0.0;
    for (int j = 0; j <= i; ++j) s = __dadd_rn(s, __dmul_rn(GM(L, i, j), v[j]));
    tmp[i] = s;
  }
  __syncwarp();
  for (int i = lane; i < d; i += 32) v[i] = tmp[i];
  __syncwarp();
}

// augur_mat_mvm (:412-420): dst = A v.
__device__ void w_mvm(double* dst, const double* A, const double* v, int d) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < d; i += 32) {
    double s = 0.0;
    for (int j = 0; j < d; ++j) s = __dadd_rn(s, __dmul_rn(GM(A, i, j), v[j]));
    dst[i] = s;
  }
  __syncwarp();
}

// augur_mat_trtrmm (:381-392): L2 = L1 L2 (rows below i are original when row
// i is formed).
__device__ void w_trtrmm(const double* L1, double* L2, double* tmp, int d) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < d * d; e += 32) {
    const int i = e / d, j = e - i * d;
    double s = 0.0;
    for (int k = 0; k < i; ++k) s = __dadd_rn(s, __dmul_rn(GM(L1, i, k), GM(L2, k, j)));
    s = __dadd_rn(s, __dmul_rn(GM(L1, i, i), GM(L2, i, j)));
    tmp[e] = s;
  }
  __syncwarp();
  for (int e = lane; e < d * d; e += 32) L2[e] = tmp[e];
  __syncwarp();
}

// augur_mvnormal_sample (augur_dist.c:622-630): the d normals at positions
// s.pos .. s.pos+d-1 of the stream (the caller advances its cursor by d),
// then chol(cov) v + mean.  L, tmp: scratch.
__device__ void w_mvn_sample(const Stream& s, double* result, const double* mean, const double* cov, double* L,
                             double* tmp, int d) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < d; i += 32) {
    Stream si = s;
    si.pos = s.pos + (uint32_t)i;
    result[i] = si.normal();
  }
  for (int e = lane; e < d * d; e += 32) L[e] = cov[e];
  __syncwarp();
  w_chol(L, d);
  w_trvm(L, result, tmp, d);
  for (int i = lane; i < d; i += 32) result[i] = __dadd_rn(result[i], mean[i]);
  __syncwarp();
}

// ---- per-component tables for the assignment draw -------------------------
// Linv = lower_trmi(chol(cov_k)) and hdet = 0.5 * log((prod L_ii)^2), the
// quantities augur_mvnormal_ll (augur_dist.c:548-568) derives from cov.
__global__ void __launch_bounds__(32)
gmm_prep_kernel(int d, const double* __restrict__ cov, double* __restrict__ Linv, double* __restrict__ hdet) {
  extern __shared__ double sm[];
  const int k = blockIdx.x;
  double* L = sm;
  double* T = sm + d * d;
  const int lane = threadIdx.x;
  for (int e = lane; e < d * d; e += 32) L[e] = cov[(size_t)k * d * d + e];
  __syncwarp();
  w_chol(L, d);
  if (lane == 0) {
    double det = 1.0;
    for (int i = 0; i < d; ++i) det = __dmul_rn(det, GM(L, i, i));
    det = __dmul_rn(det, det);
    hdet[k] = __dmul_rn(0.5, log(det));
  }
  __syncwarp();
  w_trmi(L, T, d);
  for (int e = lane; e < d * d; e += 32) Linv[(size_t)k * d * d + e] = L[e];
}

// ---- assignment draw --------------------------------------------------------
// One thread per point.  For each component: w = y - mu_k; w' = Linv w
// (ascending j per row); expon = sum_i w'_i^2; ll = c - hdet - expon/2;
// pmf_k = (1 * pis_k) * exp(ll) (CgDisc.hs:132-139); then the unnormalised
// discrete draw of augur_dist.c:798-813 with the uniform of substream
// (n, iter, 1|comp<<8).
template <int DT, bool UNROLL>
__global__ void __launch_bounds__(GMM_THREADS, 3)   // 3 CTAs per SM: measured 6 % faster than 1 at d = 32
gmm_z_kernel(int N, int d, int K, int shared_cov, const float* __restrict__ Y, const double* __restrict__ pis,
             const double* __restrict__ mu, const double* __restrict__ Linv, const double* __restrict__ hdet,
             int* __restrict__ z, uint64_t seed, uint32_t iter, uint32_t comp) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const double c = __dmul_rn(__dmul_rn(-0.5, (double)d), log(2.0 * 3.14159265358979323846264338327950288));
  double y[DT], w[DT];
#pragma unroll
  for (int i = 0; i < DT; ++i) y[i] = i < d ? (double)Y[(size_t)n * d + i] : 0.0;
  static_assert(UNROLL || DT == GMM_MAX_D, "generic path is the widest");
  double pmf[GMM_MAX_K];
  for (int k = 0; k < K; ++k) {
    const int kc = shared_cov ? 0 : k;
    const double* Lk = Linv + (size_t)kc * d * d;
    const double* mk = mu + (size_t)k * d;
#pragma unroll
    for (int i = 0; i < DT; ++i) w[i] = i < d ? __dadd_rn(y[i], -__ldg(mk + i)) : 0.0;
    double expon = 0.0;
#pragma unroll
    for (int i = 0; i < DT; ++i) {
      if (i < d) {
        double s = 0.0;
        if (UNROLL) {
#pragma unroll
          for (int j = 0; j <= i; ++j) s = __dadd_rn(s, __dmul_rn(__ldg(Lk + (size_t)i * d + j), w[j]));
        } else {
          for (int j = 0; j <= i; ++j) s = __dadd_rn(s, __dmul_rn(__ldg(Lk + (size_t)i * d + j), w[j]));
        }
        expon = __dadd_rn(expon, __dmul_rn(s, s));
      }
    }
    const double ll = __dadd_rn(__dadd_rn(c, -__ldg(hdet + kc)), -__dmul_rn(0.5, expon));
    double prob = 1.0;
    prob = __dmul_rn(prob, __ldg(pis + k));
    prob = __dmul_rn(prob, exp(ll));
    pmf[k] = prob;
  }
  Stream s = make_stream(seed, (uint32_t)n, iter, TAG_Z | (comp << 8));
  const double u = s.uniform();
  double norm = 0.0;
  for (int k = 0; k < K; ++k) norm = __dadd_rn(norm, pmf[k]);
  double acc = __ddiv_rn(pmf[0], norm);
  int zk = K - 1;
  for (int i = 1; i < K; ++i) {
    if (u < acc) { zk = i - 1; break; }
    acc = __dadd_rn(acc, __ddiv_rn(pmf[i], norm));
  }
  z[n] = zk;
}

// ---- conjugate statistics ----------------------------------------------------
// CTA b accumulates points [b*chunk, (b+1)*chunk): counts, sum of y
// (want_sum) and the lower triangle of sum (y - mu_z)(y - mu_z)^T
// (want_obs; the reference's full-matrix update augur_mat_atm_inc_vtmt is
// symmetric elementwise).  The chunk is taken in sub-chunks of at most
// `sub` points: a sub-chunk's rows of Y are copied to shared memory with
// coalesced loads (all in flight at once), sorted by component with a
// stable counting sort (warp 0, match_any ranks), and the components are
// walked one at a time: each thread owns fixed table entries and
// accumulates them in registers over the component's points in point order,
// adding the sub-chunk's sum to its partial.  Partials go to scratch
// [CTA][K][W] and gmm_stats_reduce_kernel adds them in CTA order
// (deterministic; the reference adds in point order).
constexpr int GMM_STAT_MAXE = 4;       // table entries per thread (W <= 4 * GMM_THREADS)
constexpr int GMM_STAT_SMEM = 96 * 1024;

__host__ __device__ inline int gmm_stat_sub(int d, int chunk) {
  const int fit = GMM_STAT_SMEM / (4 * d + 8);
  return chunk < fit ? chunk : fit;
}

__global__ void __launch_bounds__(GMM_THREADS)
gmm_stats_kernel(int N, int d, int K, const float* __restrict__ Y, const int* __restrict__ z,
                 const double* __restrict__ mu, int want_sum, int want_obs, int chunk,
                 double* __restrict__ part) {
  extern __shared__ int sidx[];          // zs [sub], perm [sub], ys [sub][d] (float)
  __shared__ int koff[GMM_MAX_K + 1];
  const int sub = gmm_stat_sub(d, chunk);
  int* zs = sidx;
  int* perm = sidx + sub;
  float* ys = reinterpret_cast<float*>(sidx + 2 * sub);
  const int T = d * (d + 1) / 2;
  const int W = 1 + (want_sum ? d : 0) + (want_obs ? T : 0);
  const int tid = threadIdx.x, lane = tid & 31;
  const int n0 = blockIdx.x * chunk, n1 = min(N, n0 + chunk);
  // entries owned by this thread: kind 0 count, 1 sum of y_i, 2 scatter (i, j)
  int ekind[GMM_STAT_MAXE], ei[GMM_STAT_MAXE], ej[GMM_STAT_MAXE];
  int ne = 0;
  for (int e = tid; e < W && ne < GMM_STAT_MAXE; e += blockDim.x, ++ne) {
    if (e == 0) { ekind[ne] = 0; ei[ne] = 0; ej[ne] = 0; }
    else if (want_sum && e <= d) { ekind[ne] = 1; ei[ne] = e - 1; ej[ne] = 0; }
    else {
      int t = e - 1 - (want_sum ? d : 0);
      int i = 0;
      while (t >= i + 1) { t -= i + 1; ++i; }
      ekind[ne] = 2; ei[ne] = i; ej[ne] = t;
    }
  }
  for (int base = n0; base < n1 || base == n0; base += sub) {
    const int m = max(0, min(sub, n1 - base));
    for (int p = tid; p < m; p += blockDim.x) {
      const int k = z[base + p];
      zs[p] = (k >= 0 && k < K) ? k : -1;    // a label outside [0, K) is not counted
    }
    for (int e = tid; e < m * d; e += blockDim.x) ys[e] = Y[(size_t)base * d + e];
    __syncthreads();
    if (tid < 32) {
      // stable counting sort of the sub-chunk by component
      for (int k = lane; k <= K; k += 32) koff[k] = 0;
      __syncwarp();
      for (int p = lane; p < m; p += 32)
        if (zs[p] >= 0) atomicAdd(&koff[zs[p] + 1], 1);
      __syncwarp();
      if (lane == 0)
        for (int k = 0; k < K; ++k) koff[k + 1] += koff[k];
      __syncwarp();
      for (int p0 = 0; p0 < m; p0 += 32) {       // koff[k] serves as component k's cursor
        const int p = p0 + lane;
        const int k = p < m ? zs[p] : -1;
        const bool act = k >= 0;
        const unsigned mask = __ballot_sync(0xffffffffu, act);
        if (act) {
          const unsigned peers = __match_any_sync(mask, k);
          const int rank = __popc(peers & ((1u << lane) - 1u));
          perm[koff[k] + rank] = p;
          __syncwarp(mask);
          if (lane == __ffs(peers) - 1) koff[k] += __popc(peers);
        }
        __syncwarp();
      }
      if (lane == 0) {                           // cursors back to start offsets
        for (int k = K; k > 0; --k) koff[k] = koff[k - 1];
        koff[0] = 0;
      }
    }
    __syncthreads();
    for (int k = 0; k < K; ++k) {
      double acc[GMM_STAT_MAXE], mi[GMM_STAT_MAXE], mj[GMM_STAT_MAXE];
#pragma unroll
      for (int q = 0; q < GMM_STAT_MAXE; ++q) {
        acc[q] = 0.0;
        mi[q] = (q < ne && ekind[q] == 2) ? mu[(size_t)k * d + ei[q]] : 0.0;
        mj[q] = (q < ne && ekind[q] == 2) ? mu[(size_t)k * d + ej[q]] : 0.0;
      }
      for (int p = koff[k]; p < koff[k + 1]; ++p) {
        const float* y = ys + perm[p] * d;
#pragma unroll
        for (int q = 0; q < GMM_STAT_MAXE; ++q) {
          if (q < ne) {
            if (ekind[q] == 0) {
              acc[q] = __dadd_rn(acc[q], 1.0);
            } else if (ekind[q] == 1) {
              acc[q] = __dadd_rn(acc[q], (double)y[ei[q]]);
            } else {
              const double di = __dadd_rn((double)y[ei[q]], -mi[q]);
              const double dj = __dadd_rn((double)y[ej[q]], -mj[q]);
              acc[q] = __dadd_rn(acc[q], __dmul_rn(di, dj));
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < GMM_STAT_MAXE; ++q) {
        if (q < ne) {
          double* dst = part + ((size_t)blockIdx.x * K + k) * W + tid + q * blockDim.x;
          *dst = base == n0 ? acc[q] : __dadd_rn(*dst, acc[q]);
        }
      }
    }
    __syncthreads();                             // the next sub-chunk reuses shared memory
    if (m == 0) break;
  }
}

__global__ void gmm_stats_reduce_kernel(int d, int K, int want_sum, int want_obs, int nparts,
                                        const double* __restrict__ part, int* __restrict__ cnt,
                                        double* __restrict__ sum, double* __restrict__ obs) {
  const int T = d * (d + 1) / 2;
  const int W = 1 + (want_sum ? d : 0) + (want_obs ? T : 0);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K * W) return;
  // CTA-order sum; eight partials are loaded ahead of their additions
  double a = 0.0;
  const size_t stride = (size_t)K * W;
  int b = 0;
  for (; b + 8 <= nparts; b += 8) {
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = __ldg(part + (size_t)(b + q) * stride + e);
#pragma unroll
    for (int q = 0; q < 8; ++q) a = __dadd_rn(a, v[q]);
  }
  for (; b < nparts; ++b) a = __dadd_rn(a, __ldg(part + (size_t)b * stride + e));
  const int k = e / W, f = e - k * W;
  if (f == 0) {
    cnt[k] = (int)a;
  } else if (want_sum && f <= d) {
    sum[(size_t)k * d + f - 1] = a;
  } else {
    int t = f - 1 - (want_sum ? d : 0);
    int i = 0;
    while (t >= i + 1) { t -= i + 1; ++i; }
    obs[(size_t)k * d * d + (size_t)i * d + t] = a;
    obs[(size_t)k * d * d + (size_t)t * d + i] = a;
  }
}

// ---- conjugate draws -----------------------------------------------------------
// Dirichlet(alpha + cnt) for the weights (augur_dist.c:526-538), element
// substream (k, iter, 7|comp<<8); sequential normaliser.
__global__ void gmm_conj_pis_kernel(int K, const double* __restrict__ alpha, const int* __restrict__ cnt,
                                    double* __restrict__ pis, uint64_t seed, uint32_t iter, uint32_t comp) {
  __shared__ double g[GMM_MAX_K];
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    Stream s = make_stream(seed, (uint32_t)k, iter, TAG_PI | (comp << 8));
    g[k] = gamma_draw(s, __dadd_rn(alpha[k], (double)cnt[k]), 1.0);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double acc = 0.0;
    for (int k = 0; k < K; ++k) acc = __dadd_rn(acc, g[k]);
    for (int k = 0; k < K; ++k) pis[k] = __ddiv_rn(g[k], acc);
  }
}

// augur_mvnormal_mvnormal_conj (augur_dist.c:633-669) for component k, one
// warp, substream (k, iter, 8|comp<<8).
__global__ void __launch_bounds__(64)
gmm_conj_mu_kernel(int d, int shared_cov, const double* __restrict__ mu0, const double* __restrict__ cov0,
                   const int* __restrict__ cnt, const double* __restrict__ sum, const double* __restrict__ cov,
                   double* __restrict__ mu, uint64_t seed, uint32_t iter, uint32_t comp) {
  extern __shared__ double sm[];
  const int k = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int dd = d * d;
  double* L0 = sm;
  double* L = L0 + dd;
  double* T = L + dd;
  double* T2 = T + dd;
  double* res = T2 + dd;
  double* w0 = res + d;
  double* mean = w0 + d;
  double* sk = mean + d;
  double* tmp = sk + d;
  double* mu0s = tmp + d;
  const double* ck = cov + (size_t)(shared_cov ? 0 : k) * dd;
  for (int e = threadIdx.x; e < dd; e += blockDim.x) { L0[e] = cov0[e]; L[e] = ck[e]; }
  for (int i = threadIdx.x; i < d; i += blockDim.x) { sk[i] = sum[(size_t)k * d + i]; mu0s[i] = mu0[i]; }
  __syncthreads();
  // the two inverses are independent: one warp each (each the reference's
  // sequential routine, so the values are unchanged), then warp 0 alone
  if (warp == 0) {
    w_chol(L0, d);
    w_cholinv(L0, T, d);
  } else {
    w_chol(L, d);
    w_cholinv(L, T2, d);
  }
  __syncthreads();
  if (warp != 0) return;
  const int n = cnt[k];
  for (int e = lane; e < dd; e += 32) L[e] = __dmul_rn((double)n, L[e]);           // augur_mat_ms
  __syncwarp();
  w_mvm(res, L0, mu0s, d);
  const double sc = n == 0 ? 1.0 : __ddiv_rn(1.0, (double)n);                       // augur_vec_scale
  for (int i = lane; i < d; i += 32) sk[i] = __dmul_rn(sc, sk[i]);
  __syncwarp();
  w_mvm(w0, L, sk, d);
  for (int i = lane; i < d; i += 32) res[i] = __dadd_rn(res[i], w0[i]);
  for (int e = lane; e < dd; e += 32) L0[e] = __dadd_rn(L0[e], L[e]);              // augur_mat_plus
  __syncwarp();
  w_chol(L0, d);
  w_cholinv(L0, T, d);
  w_mvm(mean, L0, res, d);
  const Stream s = make_stream(seed, (uint32_t)k, iter, TAG_MU | (comp << 8));
  w_mvn_sample(s, res, mean, L0, L, tmp, d);
  for (int i = lane; i < d; i += 32) mu[(size_t)k * d + i] = res[i];
}

// Bartlett diagonal for the inverse-Wishart draw (bartlett_decomp,
// augur_dist.c:722-738): the chi-square of n - i degrees of freedom in row i
// is the sum of squares of the n - i normals at stream positions
// i*n + i + t, t < n - i (n = cnt[k] + df), substream (k, iter, 9|comp<<8).
// One CTA per (k, i): thread-strided partial sums, then the fixed-order
// block sum.  That is O(d * cnt[k]) normals per component per sweep (the
// reference's algorithm), spread over K * d CTAs.  The sums are staged on
// the diagonal of cov[k], which gmm_conj_cov_kernel then reads and
// overwrites with the draw.
__global__ void __launch_bounds__(GMM_THREADS)
gmm_bartlett_chi_kernel(int d, int df, const int* __restrict__ cnt, double* __restrict__ cov, uint64_t seed,
                        uint32_t iter, uint32_t comp) {
  __shared__ double red[34];
  const int k = blockIdx.x / d, i = blockIdx.x - k * d;
  const int n = cnt[k] + df;
  const Stream s0 = make_stream(seed, (uint32_t)k, iter, TAG_COV | (comp << 8));
  double local = 0.0;
  for (int t = threadIdx.x; t < n - i; t += blockDim.x) {
    Stream s = s0;
    s.pos = (uint32_t)(i * n + i + t);
    const double zz = s.normal();
    local = __dadd_rn(local, __dmul_rn(zz, zz));
  }
  const double chi = block_sum_f64(local, red);
  if (threadIdx.x == 0) cov[(size_t)k * d * d + (size_t)i * d + i] = chi;
}

// augur_invwishart_mvnormal_conj (augur_dist.c:751-757) and
// augur_invwishart_sample (:740-749) with bartlett_decomp (:722-738) for
// component k, one thread block, substream (k, iter, 9|comp<<8).  The
// Bartlett normals are drawn at the stream positions the reference's loop
// consumes them (row-major over the lower triangle; each diagonal
// chi-square of n - i normals follows its row's off-diagonal normals).  The
// chi-square sums of up to cnt + df squares come from
// gmm_bartlett_chi_kernel (on cov's diagonal), added in a fixed tree order
// instead of sequentially (a rounding-level difference); the d x d algebra
// runs on warp 0.
__global__ void __launch_bounds__(GMM_THREADS)
gmm_conj_cov_kernel(int d, int df, const double* __restrict__ scale0, const int* __restrict__ cnt,
                    const double* __restrict__ obs, double* __restrict__ cov, uint64_t seed, uint32_t iter,
                    uint32_t comp) {
  extern __shared__ double sm[];
  const int k = blockIdx.x, tid = threadIdx.x;
  const int dd = d * d;
  double* S = sm;          // obs + scale0
  double* L = S + dd;
  double* A = L + dd;
  double* T = A + dd;
  for (int e = tid; e < dd; e += blockDim.x) {
    S[e] = __dadd_rn(obs[(size_t)k * dd + e], scale0[e]);
    L[e] = S[e];
  }
  __syncthreads();
  const int n = cnt[k] + df;
  if (tid < 32) {
    w_chol(L, d);
    w_cholinv(L, T, d);
    w_chol(L, d);
  }
  // Bartlett factor: element (i, j < i) is the normal at position i*n + j;
  // the diagonal (i, i) is the square root of the row's chi-square sum.
  const Stream s0 = make_stream(seed, (uint32_t)k, iter, TAG_COV | (comp << 8));
  for (int e = tid; e < dd; e += blockDim.x) {
    const int i = e / d, j = e - i * d;
    if (j < i) {
      Stream s = s0;
      s.pos = (uint32_t)(i * n + j);
      A[e] = s.normal();
    } else if (j > i) {
      A[e] = 0.0;
    } else {
      A[e] = __dsqrt_rn(cov[(size_t)k * dd + e]);
    }
  }
  __syncthreads();
  if (tid < 32) {
    w_trtrmm(L, A, T, d);
    w_cholinv(A, T, d);
  }
  __syncthreads();
  for (int e = tid; e < dd; e += blockDim.x) cov[(size_t)k * dd + e] = A[e];
}

// ---- ESlice / MWG on the means ---------------------------------------------------
// Full conditional of mu[k] (CgLike.hs:236-265): its prior MvNormal(mu0,
// cov0) plus the points of component k, evaluated by the whole CTA at the
// candidate in shared memory `cand`.  The per-point terms use the per-sweep
// Linv/hdet tables of component k; the prior uses its own table (slot Kc).
__device__ double cta_mvn_ll_point(const double* y, const double* m, const double* Li, double hdet, int d) {
  const double c = __dmul_rn(__dmul_rn(-0.5, (double)d), log(2.0 * 3.14159265358979323846264338327950288));
  double expon = 0.0;
  for (int i = 0; i < d; ++i) {
    double s = 0.0;
    for (int j = 0; j <= i; ++j) s = __dadd_rn(s, __dmul_rn(Li[(size_t)i * d + j], __dadd_rn(y[j], -m[j])));
    expon = __dadd_rn(expon, __dmul_rn(s, s));
  }
  return __dadd_rn(__dadd_rn(c, -hdet), -__dmul_rn(0.5, expon));
}

__device__ double cta_ll_mu(int N, int d, int k, int kc, const float* __restrict__ Y, const int* __restrict__ z,
                            const double* cand, const double* mu0, const double* Linv, const double* hdet,
                            int prior_slot, double* red, double* ybuf) {
  double local = 0.0;
  double* yt = ybuf + (size_t)threadIdx.x * GMM_MAX_D;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    if (z[n] != k) continue;
    for (int i = 0; i < d; ++i) yt[i] = (double)Y[(size_t)n * d + i];
    local = __dadd_rn(local, cta_mvn_ll_point(yt, cand, Linv + (size_t)kc * d * d, hdet[kc], d));
  }
  const double data = block_sum_f64(local, red);
  // prior MvNormal(cand; mu0, cov0): point cand, mean mu0
  const double prior = cta_mvn_ll_point(cand, mu0, Linv + (size_t)prior_slot * d * d, hdet[prior_slot], d);
  double ll = 0.0;
  ll = __dadd_rn(ll, prior);
  ll = __dadd_rn(ll, data);
  return ll;
}

// augur_mcmc_eslice (augur_mcmclib.h:439-485) on mu[k]; substream
// (k, iter, 10|comp<<8): nu (d normals), u, theta, one uniform per shrink.
// Warp 0 does the small vector work, the CTA evaluates log-densities.
__global__ void __launch_bounds__(GMM_THREADS)
gmm_eslice_kernel(int N, int d, int shared_cov, const float* __restrict__ Y, const int* __restrict__ z,
                  const double* __restrict__ mu0, const double* __restrict__ cov0, const double* __restrict__ Linv,
                  const double* __restrict__ hdet, int prior_slot, double* __restrict__ mu, uint64_t seed,
                  uint32_t iter, uint32_t comp, int* __restrict__ shrinks) {
  extern __shared__ double sm[];
  const int k = blockIdx.x, kc = shared_cov ? 0 : k;
  const int dd = d * d;
  double* cur = sm;
  double* nu = cur + d;
  double* prop = nu + d;
  double* mu0s = prop + d;
  double* L = mu0s + d;
  double* tmp = L + dd;
  double* red = tmp + d;
  double* bc = red + 34;
  double* ybuf = bc + 8;
  for (int i = threadIdx.x; i < d; i += blockDim.x) { cur[i] = mu[(size_t)k * d + i]; mu0s[i] = mu0[i]; }
  __syncthreads();
  Stream s = make_stream(seed, (uint32_t)k, iter, TAG_ESLICE | (comp << 8));
  if (threadIdx.x < 32) w_mvn_sample(s, nu, mu0s, cov0, L, tmp, d);
  s.pos += (uint32_t)d;   // every thread advances the same cursor
  __syncthreads();
  const double PI2 = 2.0 * 3.14159265358979323846264338327950288;
  const double u = s.uniform();
  const double lcur = cta_ll_mu(N, d, k, kc, Y, z, cur, mu0s, Linv, hdet, prior_slot, red, ybuf);
  const double log_y = __dadd_rn(lcur, log(u));
  double theta = __dadd_rn(0.0, __dmul_rn(s.uniform(), __dadd_rn(PI2, -0.0)));
  double tmin = __dadd_rn(theta, -PI2), tmax = theta;
  int ns = 0;
  for (int guard = 0; guard < 2000; ++guard) {
    const double diff = __dadd_rn(tmax, -tmin);
    if (diff < 1e-8) break;
    const double ct = cos(theta), st = sin(theta);
    for (int i = threadIdx.x; i < d; i += blockDim.x) {
      const double mi = mu0s[i];
      const double a = __dmul_rn(__dadd_rn(cur[i], -mi), ct);
      const double b = __dmul_rn(__dadd_rn(nu[i], -mi), st);
      prop[i] = __dadd_rn(__dadd_rn(a, b), mi);
    }
    __syncthreads();
    const double pll = cta_ll_mu(N, d, k, kc, Y, z, prop, mu0s, Linv, hdet, prior_slot, red, ybuf);
    if (pll > log_y) {
      for (int i = threadIdx.x; i < d; i += blockDim.x) cur[i] = prop[i];
      __syncthreads();
      break;
    }
    if (theta < 0) tmin = theta; else tmax = theta;
    theta = __dadd_rn(tmin, __dmul_rn(s.uniform(), __dadd_rn(tmax, -tmin)));
    ++ns;
  }
  for (int i = threadIdx.x; i < d; i += blockDim.x) mu[(size_t)k * d + i] = cur[i];
  if (threadIdx.x == 0) shrinks[k] = ns;
}

// MWG [mu] ~ MvNormal(mu[k], covp) (CgUserProp.hs:131-260 over
// augur_mcmc_mwg); compat uses the generated log-correction
// ll(mu; mu, covp) - ll(mu'; mu, covp), else 0.  Substream (k, iter,
// 11|comp<<8): d normals, then the accept uniform.  Linv slot `prop_slot`
// holds the proposal covariance's table.
__global__ void __launch_bounds__(GMM_THREADS)
gmm_mwg_kernel(int N, int d, int shared_cov, const float* __restrict__ Y, const int* __restrict__ z,
               const double* __restrict__ mu0, const double* __restrict__ covp, const double* __restrict__ Linv,
               const double* __restrict__ hdet, int prior_slot, int prop_slot, int compat,
               double* __restrict__ mu, uint64_t seed, uint32_t iter, uint32_t comp, int* __restrict__ accepts) {
  extern __shared__ double sm[];
  const int k = blockIdx.x, kc = shared_cov ? 0 : k;
  const int dd = d * d;
  double* cur = sm;
  double* prop = cur + d;
  double* mu0s = prop + d;
  double* L = mu0s + d;
  double* tmp = L + dd;
  double* red = tmp + d;
  double* bc = red + 34;
  double* ybuf = bc + 8;
  for (int i = threadIdx.x; i < d; i += blockDim.x) { cur[i] = mu[(size_t)k * d + i]; mu0s[i] = mu0[i]; }
  __syncthreads();
  Stream s = make_stream(seed, (uint32_t)k, iter, TAG_MWG | (comp << 8));
  if (threadIdx.x < 32) w_mvn_sample(s, prop, cur, covp, L, tmp, d);
  s.pos += (uint32_t)d;
  __syncthreads();
  double corr = 0.0;
  if (compat) {
    corr = __dadd_rn(cta_mvn_ll_point(cur, cur, Linv + (size_t)prop_slot * dd, hdet[prop_slot], d),
                     -cta_mvn_ll_point(prop, cur, Linv + (size_t)prop_slot * dd, hdet[prop_slot], d));
  }
  const double cl = cta_ll_mu(N, d, k, kc, Y, z, cur, mu0s, Linv, hdet, prior_slot, red, ybuf);
  const double pl = cta_ll_mu(N, d, k, kc, Y, z, prop, mu0s, Linv, hdet, prior_slot, red, ybuf);
  const double u = s.uniform();
  const int acc = log(u) < __dadd_rn(__dadd_rn(pl, -cl), corr);
  if (acc)
    for (int i = threadIdx.x; i < d; i += blockDim.x) mu[(size_t)k * d + i] = prop[i];
  if (threadIdx.x == 0) accepts[k] += acc;
}

#undef GM

// ---- launchers -------------------------------------------------------------------
static int gmm_check(int N, int d, int K) {
  AB_REQUIRE(N > 0 && d > 0 && d <= GMM_MAX_D && K > 0 && K <= GMM_MAX_K, AB_ERR_ARG,
             "gmm: need N > 0, 0 < d <= %d, 0 < K <= %d (N=%d d=%d K=%d)", GMM_MAX_D, GMM_MAX_K, N, d, K);
  return AB_OK;
}

template <int DT, bool U>
static void launch_z_t(int N, int d, int K, int shared, const float* Y, const double* pis, const double* mu,
                       const double* Linv, const double* hdet, int* z, uint64_t seed, uint32_t iter,
                       uint32_t comp, cudaStream_t st) {
  gmm_z_kernel<DT, U><<<ceil_div(N, GMM_THREADS), GMM_THREADS, 0, st>>>(N, d, K, shared, Y, pis, mu, Linv, hdet,
                                                                     z, seed, iter, comp);
}

int launch_gmm_z(int N, int d, int K, int shared, const float* Y, const double* pis, const double* mu,
                 const double* Linv, const double* hdet, int* z, uint64_t seed, uint32_t iter, uint32_t comp,
                 cudaStream_t st) {
  if (d <= 2) launch_z_t<2, true>(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, iter, comp, st);
  else if (d <= 4) launch_z_t<4, true>(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, iter, comp, st);
  else if (d <= 8) launch_z_t<8, true>(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, iter, comp, st);
  else if (d <= 16) launch_z_t<16, true>(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, iter, comp, st);
  else if (d <= 32) launch_z_t<32, true>(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, iter, comp, st);
  else launch_z_t<GMM_MAX_D, false>(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, iter, comp, st);
  AB_LAUNCH_CHECK("gmm_z_kernel");
  return AB_OK;
}

int launch_gmm_prep(int Kc, int d, const double* cov, double* Linv, double* hdet, cudaStream_t st) {
  const size_t smem = sizeof(double) * 2 * (size_t)d * d;
  AB_CUDA(cudaFuncSetAttribute(gmm_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_prep_kernel<<<Kc, 32, smem, st>>>(d, cov, Linv, hdet);
  AB_LAUNCH_CHECK("gmm_prep_kernel");
  return AB_OK;
}

size_t gmm_stats_scratch(int d, int K) {
  const size_t W = 1 + (size_t)d + (size_t)d * (d + 1) / 2;
  return sizeof(double) * GMM_STAT_CTAS * (size_t)K * W;
}

int launch_gmm_stats(int N, int d, int K, const float* Y, const int* z, const double* mu, int want_sum,
                     int want_obs, int* cnt, double* sum, double* obs, double* part, cudaStream_t st) {
  const int T = d * (d + 1) / 2;
  const int W = 1 + (want_sum ? d : 0) + (want_obs ? T : 0);
  AB_REQUIRE(W <= GMM_STAT_MAXE * GMM_THREADS, AB_ERR_ARG, "gmm: d too large for the statistics pass");
  const int chunk = (N + GMM_STAT_CTAS - 1) / GMM_STAT_CTAS;
  const int nparts = (N + chunk - 1) / chunk;
  const int sub = gmm_stat_sub(d, chunk);
  const size_t smem = (sizeof(int) * 2 + sizeof(float) * (size_t)d) * (size_t)sub;
  AB_CUDA(cudaFuncSetAttribute(gmm_stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_stats_kernel<<<nparts, GMM_THREADS, smem, st>>>(N, d, K, Y, z, mu, want_sum, want_obs, chunk, part);
  AB_LAUNCH_CHECK("gmm_stats_kernel");
  gmm_stats_reduce_kernel<<<ceil_div((size_t)K * W, 256), 256, 0, st>>>(d, K, want_sum, want_obs, nparts, part,
                                                                        cnt, sum, obs);
  AB_LAUNCH_CHECK("gmm_stats_reduce_kernel");
  return AB_OK;
}

int launch_gmm_conj_mu(int K, int d, int shared, const double* mu0, const double* cov0, const int* cnt,
                       const double* sum, const double* cov, double* mu, uint64_t seed, uint32_t iter,
                       uint32_t comp, cudaStream_t st) {
  const size_t smem = sizeof(double) * (4 * (size_t)d * d + 6 * (size_t)d);
  AB_CUDA(cudaFuncSetAttribute(gmm_conj_mu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_conj_mu_kernel<<<K, 64, smem, st>>>(d, shared, mu0, cov0, cnt, sum, cov, mu, seed, iter, comp);
  AB_LAUNCH_CHECK("gmm_conj_mu_kernel");
  return AB_OK;
}

int launch_gmm_conj_cov(int K, int d, int df, const double* scale0, const int* cnt, const double* obs,
                        double* cov, uint64_t seed, uint32_t iter, uint32_t comp, cudaStream_t st) {
  gmm_bartlett_chi_kernel<<<K * d, GMM_THREADS, 0, st>>>(d, df, cnt, cov, seed, iter, comp);
  AB_LAUNCH_CHECK("gmm_bartlett_chi_kernel");
  const size_t smem = sizeof(double) * 4 * (size_t)d * d;
  AB_CUDA(cudaFuncSetAttribute(gmm_conj_cov_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_conj_cov_kernel<<<K, GMM_THREADS, smem, st>>>(d, df, scale0, cnt, obs, cov, seed, iter, comp);
  AB_LAUNCH_CHECK("gmm_conj_cov_kernel");
  return AB_OK;
}

size_t gmm_move_smem(int d) {
  return sizeof(double) * ((size_t)5 * d + (size_t)d * d + 34 + 8 + (size_t)GMM_THREADS * GMM_MAX_D);
}

}  // namespace ab

using namespace ab;

// ------------------------------- C ABI ----------------------------------------------

extern "C" size_t ab_gmm_table_doubles(int Kc, int d) { return (size_t)Kc * d * d + (size_t)Kc; }

extern "C" int ab_gmm_prep(int Kc, int d, const double* cov, double* Linv, double* hdet, void* stream) {
  AB_REQUIRE(Kc > 0 && d > 0 && d <= GMM_MAX_D, AB_ERR_ARG, "ab_gmm_prep: bad sizes");
  AB_REQUIRE(cov && Linv && hdet, AB_ERR_ARG, "ab_gmm_prep: null pointer");
  return launch_gmm_prep(Kc, d, cov, Linv, hdet, as_stream(stream));
}

extern "C" int ab_gmm_disc_z(int N, int d, int K, int shared_cov, const float* Y, const double* pis,
                             const double* mu, const double* Linv, const double* hdet, int* z, uint64_t seed,
                             uint32_t iter, uint32_t comp, void* stream) {
  int rc = gmm_check(N, d, K);
  if (rc) return rc;
  AB_REQUIRE(Y && pis && mu && Linv && hdet && z, AB_ERR_ARG, "ab_gmm_disc_z: null pointer");
  return launch_gmm_z(N, d, K, shared_cov, Y, pis, mu, Linv, hdet, z, seed, iter, comp, as_stream(stream));
}

extern "C" size_t ab_gmm_stats_scratch_bytes(int d, int K) { return gmm_stats_scratch(d, K); }

extern "C" int ab_gmm_stats(int N, int d, int K, const float* Y, const int* z, const double* mu, int* cnt,
                            double* sum, double* obs, void* scratch, void* stream) {
  int rc = gmm_check(N, d, K);
  if (rc) return rc;
  AB_REQUIRE(Y && z && cnt && scratch, AB_ERR_ARG, "ab_gmm_stats: null pointer");
  AB_REQUIRE(!obs || mu, AB_ERR_ARG, "ab_gmm_stats: the scatter matrices need mu");
  return launch_gmm_stats(N, d, K, Y, z, mu, sum != nullptr, obs != nullptr, cnt, sum, obs,
                          static_cast<double*>(scratch), as_stream(stream));
}

extern "C" int ab_gmm_conj_pis(int K, const double* alpha, const int* cnt, double* pis, uint64_t seed,
                               uint32_t iter, uint32_t comp, void* stream) {
  AB_REQUIRE(K > 0 && K <= GMM_MAX_K, AB_ERR_ARG, "ab_gmm_conj_pis: bad K");
  AB_REQUIRE(alpha && cnt && pis, AB_ERR_ARG, "ab_gmm_conj_pis: null pointer");
  gmm_conj_pis_kernel<<<1, 64, 0, as_stream(stream)>>>(K, alpha, cnt, pis, seed, iter, comp);
  AB_LAUNCH_CHECK("gmm_conj_pis_kernel");
  return AB_OK;
}

extern "C" int ab_gmm_conj_mu(int K, int d, int shared_cov, const double* mu0, const double* cov0, const int* cnt,
                              const double* sum, const double* cov, double* mu, uint64_t seed, uint32_t iter,
                              uint32_t comp, void* stream) {
  AB_REQUIRE(K > 0 && K <= GMM_MAX_K && d > 0 && d <= GMM_MAX_D, AB_ERR_ARG, "ab_gmm_conj_mu: bad sizes");
  AB_REQUIRE(mu0 && cov0 && cnt && sum && cov && mu, AB_ERR_ARG, "ab_gmm_conj_mu: null pointer");
  return launch_gmm_conj_mu(K, d, shared_cov, mu0, cov0, cnt, sum, cov, mu, seed, iter, comp, as_stream(stream));
}

extern "C" int ab_gmm_conj_cov(int K, int d, int df, const double* scale0, const int* cnt, const double* obs,
                               double* cov, uint64_t seed, uint32_t iter, uint32_t comp, void* stream) {
  AB_REQUIRE(K > 0 && K <= GMM_MAX_K && d > 0 && d <= GMM_MAX_D, AB_ERR_ARG, "ab_gmm_conj_cov: bad sizes");
  AB_REQUIRE(df > 0 && df < 100000, AB_ERR_ARG, "ab_gmm_conj_cov: bad degrees of freedom");
  AB_REQUIRE(scale0 && cnt && obs && cov, AB_ERR_ARG, "ab_gmm_conj_cov: null pointer");
  return launch_gmm_conj_cov(K, d, df, scale0, cnt, obs, cov, seed, iter, comp, as_stream(stream));
}

extern "C" int ab_gmm_eslice(int N, int d, int K, int shared_cov, const float* Y, const int* z, const double* mu0,
                             const double* cov0, const double* Linv, const double* hdet, int prior_slot,
                             double* mu, uint64_t seed, uint32_t iter, uint32_t comp, int* shrinks,
                             void* stream) {
  int rc = gmm_check(N, d, K);
  if (rc) return rc;
  AB_REQUIRE(Y && z && mu0 && cov0 && Linv && hdet && mu && shrinks, AB_ERR_ARG, "ab_gmm_eslice: null pointer");
  const size_t smem = gmm_move_smem(d);
  AB_CUDA(cudaFuncSetAttribute(gmm_eslice_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_eslice_kernel<<<K, GMM_THREADS, smem, as_stream(stream)>>>(N, d, shared_cov, Y, z, mu0, cov0, Linv, hdet,
                                                                  prior_slot, mu, seed, iter, comp, shrinks);
  AB_LAUNCH_CHECK("gmm_eslice_kernel");
  return AB_OK;
}

extern "C" int ab_gmm_mwg(int N, int d, int K, int shared_cov, const float* Y, const int* z, const double* mu0,
                          const double* covp, const double* Linv, const double* hdet, int prior_slot,
                          int prop_slot, int compat, double* mu, uint64_t seed, uint32_t iter, uint32_t comp,
                          int* accepts, void* stream) {
  int rc = gmm_check(N, d, K);
  if (rc) return rc;
  AB_REQUIRE(Y && z && mu0 && covp && Linv && hdet && mu && accepts, AB_ERR_ARG, "ab_gmm_mwg: null pointer");
  const size_t smem = gmm_move_smem(d);
  AB_CUDA(cudaFuncSetAttribute(gmm_mwg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_mwg_kernel<<<K, GMM_THREADS, smem, as_stream(stream)>>>(N, d, shared_cov, Y, z, mu0, covp, Linv, hdet,
                                                               prior_slot, prop_slot, compat, mu, seed, iter,
                                                               comp, accepts);
  AB_LAUNCH_CHECK("gmm_mwg_kernel");
  return AB_OK;
}
