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

// d <= GMM_MAX_D, so a shared-memory matrix index fits 32 bits
#define GM(A, i, j) (A)[(i) * d + (j)]

// ---- warp-level matrix routines (one full warp, matrices in shared memory)

// augur_mat_cholesky (:312-328), column by column; (i, j) uses row i and
// row j left of j, and the diagonal (j, j) - all final before column j.
// The diagonal's products A[j][k]^2 are formed on the lanes (k = lane,
// lane + 32) and every lane adds them in k order from the shuffles, so the
// sum is the reference's sequence of additions.
__device__ void w_chol(double* A, int d) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < d; ++j) {
    const double p0 = lane < j ? __dmul_rn(GM(A, j, lane), GM(A, j, lane)) : 0.0;
    const double p1 = lane + 32 < j ? __dmul_rn(GM(A, j, lane + 32), GM(A, j, lane + 32)) : 0.0;
    double sd = 0.0;
    const int j0 = j < 32 ? j : 32;
    for (int k = 0; k < j0; ++k) sd = __dadd_rn(sd, __shfl_sync(0xffffffffu, p0, k));
    for (int k = 32; k < j; ++k) sd = __dadd_rn(sd, __shfl_sync(0xffffffffu, p1, k - 32));
    const double djj = __dsqrt_rn(__dadd_rn(GM(A, j, j), -sd));
    __syncwarp();                                     // A[j][j] read by every lane before it is replaced
    if (lane == 0) GM(A, j, j) = djj;
    const double rjj = __ddiv_rn(1.0, djj);           // the reference's 1 / A[j][j], once per column
    for (int i = j + 1 + lane; i < d; i += 32) {
      double s = 0.0;
#pragma unroll 4
      for (int k = 0; k < j; ++k) s = __dadd_rn(s, __dmul_rn(GM(A, i, k), GM(A, j, k)));
      GM(A, i, j) = __dmul_rn(rjj, __dadd_rn(GM(A, i, j), -s));
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
#pragma unroll 4
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
// After trmi the factor's upper triangle is zero, so the terms k < r are
// zero products: starting from +0.0 they leave the sum +0.0, and the entry
// is the sum over k = r .. d-1 of M[k][r] M[k][c] (M the inverse factor, kept
// in T), in k order - independent of every other entry (while the entries
// are finite).  The d(d+1)/2 entries are dealt to the lanes in turn, which
// balances their d - r terms (column 0 alone used to take d^2 / 2 steps of
// one lane).
__device__ void w_cholinv(double* A, double* T, int d) {
  const int lane = threadIdx.x & 31;
  w_trmi(A, T, d);
  for (int e = lane; e < d * d; e += 32) T[e] = A[e];
  __syncwarp();
  const int ntri = d * (d + 1) / 2;
  for (int idx = lane; idx < ntri; idx += 32) {
    int r = (int)((sqrtf(8.0f * (float)idx + 1.0f) - 1.0f) * 0.5f);
    while (r * (r + 1) / 2 > idx) --r;
    while ((r + 1) * (r + 2) / 2 <= idx) ++r;
    const int c = idx - r * (r + 1) / 2;
    double acc = 0.0;
#pragma unroll 4
    for (int k = r; k < d; ++k) acc = __dadd_rn(acc, __dmul_rn(GM(T, k, r), GM(T, k, c)));
    GM(A, r, c) = acc;
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
#pragma unroll 4
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
#pragma unroll 4
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
#pragma unroll 4
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

// ---- assignment draw screened in binary32 ----------------------------------
// The same draw as gmm_z_kernel, decided for most points in binary32:
//   gmm_zs_prep_kernel  per component (once per call): the lower triangle of
//                       Linv_k and mu_k rounded to binary32, and the constants
//                       of the error bound below; log(pis_k) + c - hdet_k;
//   gmm_zs_kernel       one thread per point: t_k = log p_k in binary32 with a
//                       rigorous bound eps_k on its error against the exact
//                       value, p_k / p_max = exp(t_k - t_max), the running
//                       sums, and the reference's draw when u lies outside the
//                       sums' uncertainty band; other points go to a queue;
//   gmm_zx_kernel       one CTA per queued point, a warp per component: the
//                       reference's binary64 loop (gmm_z_kernel's operations,
//                       rows of Linv w on the lanes, every sum in its order),
//                       so every draw equals gmm_z_kernel's bit for bit.
// Error bound (u = 2^-24; all quantities of component k; L~, w~ the binary32
// values, w~_j = fl32(y_j - mu_j) with the difference formed in binary64):
//   |w~_j - w_j| <= u |w~_j| (1 + 2^-28);
//   row i of Linv w (i + 1 products, fused multiply-adds; zero padding adds
//   exact zeros): |s~_i - s_i| <= delta_i = u (1 + 4u) (i + 3) A_i,
//     A_i = sum_j |L~_ij||w~_j| <= R_i W (R_i >= ||L~_i||, W >= ||w~||);
//   expon = sum_i s_i^2: |e~ - e| <= (d + 1) u e~ + sum_i (2 |s~_i| delta_i + delta_i^2),
//     with sum_i |s~_i| a_i (a_i = (i + 3) R_i) accumulated beside the rows
//     and sum_i delta_i^2 <= u^2 (1 + 4u)^2 W^2 S_aa, S_aa = sum_i a_i^2;
//   t_k = fl(lpc_k - e~ / 2), lpc_k = fl32(log pis_k + c - hdet_k): |t_k - log p_k|
//     <= eps_k = E_k / 2 + u (|lpc_k| + |t_k|) + 2^-40 (|lpc_k| + e~ + 1) (the last
//     term covers the reference's own binary64 roundings);
//   p~_k = exp(t_k - t_max) (binary32 exp, <= 4u); the exact p_k / p_max lies
//     in [exp(dt - x), exp(dt + x)], x = eps_k + u |dt| + 4u, dt = t_k - t_max,
//     so |p~_k - p_k / p_max| <= A_k, formed with directed roundings; a
//     component far from the point has a wide band but a tiny p_k;
//   band = sum_k A_k + (K + 6) u norm~ + 2^-40 norm~ covers the running sums'
//     and u * norm's roundings, the comparisons' and the reference's running
//     quotient sums.
// A draw is decided (and equals the reference's) when u norm~ + band is below
// the first running sum that exceeds it minus band, and the previous sum plus
// band is below u norm~ - band.  Points whose largest log density is
// outside [-690, 690] (where the reference's binary64 exp could underflow or
// overflow), any non-finite value, or a call whose components have
// c - hdet_k > 700, take the exact path.
constexpr int GMM_ZS_MAXK = 32;
constexpr int GMM_ZS_THREADS = 128;

// Per component, floats: L~ with row i padded to whole float4s (zeros) at
// gmm_zs_row(i), a [d], then lpc, S_aa; the stride is whole float4s.
__host__ __device__ constexpr int gmm_zs_row(int i) { return 4 * (i / 4 + 1) * (2 * (i / 4) + i % 4); }
__host__ __device__ inline int gmm_zs_stride(int d) { return (gmm_zs_row(d) + d + 2 + 3) / 4 * 4; }

// tab: K float tables of gmm_zs_stride(d), then the means, binary64 [K][d].
__global__ void __launch_bounds__(64) gmm_zs_prep_kernel(int d, int K, int shared_cov, const double* __restrict__ pis,
                                                         const double* __restrict__ mu,
                                                         const double* __restrict__ Linv,
                                                         const double* __restrict__ hdet, float* __restrict__ tab,
                                                         int* __restrict__ flag) {
  __shared__ double red[1][64];
  const int k = blockIdx.x, kc = shared_cov ? 0 : k;
  const double* Lk = Linv + (size_t)kc * d * d;
  const double* mk = mu + (size_t)k * d;
  float* t = tab + (size_t)k * gmm_zs_stride(d);
  const int T = gmm_zs_row(d);
  float* L32 = t;
  float* a = t + T;
  float* sc = a + d;
  for (int i = threadIdx.x; i < d; i += blockDim.x) {
    double r2 = 0.0;
    const int row = gmm_zs_row(i), len = (i / 4 + 1) * 4;
    for (int j = 0; j < len; ++j) {
      const float l = j <= i ? __double2float_rn(Lk[(size_t)i * d + j]) : 0.0f;
      L32[row + j] = l;
      r2 += (double)l * (double)l;
    }
    // rounded up, with a relative slack for the binary64 sums' own rounding
    a[i] = __fmul_ru((float)(i + 3), __double2float_ru(sqrt(r2) * (1.0 + 1e-12)));
    reinterpret_cast<double*>(tab + (size_t)K * gmm_zs_stride(d))[(size_t)k * d + i] = mk[i];
  }
  __syncthreads();
  double saa = 0.0;
  for (int i = threadIdx.x; i < d; i += blockDim.x) saa += (double)a[i] * a[i];
  red[0][threadIdx.x] = saa;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)blockDim.x; ++i) saa += red[0][i];
    const double c = -0.5 * (double)d * log(2.0 * 3.14159265358979323846264338327950288);
    const double llc = c - hdet[kc];
    const double pk = pis[k];
    sc[0] = pk > 0.0 ? __double2float_rn(log(pk) + llc) : -INFINITY;
    sc[1] = __double2float_ru(saa * (1.0 + 1e-12));
    if (!(pk >= 0.0) || !(llc <= 700.0) || !isfinite(llc)) atomicExch(flag, 1);
  }
}

template <int DT>
__global__ void __launch_bounds__(GMM_ZS_THREADS, 5)   // 5 CTAs of 43 KB per SM
gmm_zs_kernel(int N, int d, int K, const float* __restrict__ Y, const double* __restrict__ mu,
              const float* __restrict__ tab,
              const int* __restrict__ flag, int* __restrict__ queue, int* __restrict__ qn, int* __restrict__ z,
              uint64_t seed, uint32_t iter, uint32_t comp) {
  extern __shared__ float ts[];   // the K components' tables, then the binary64 means
  const int stride = gmm_zs_stride(d);
  {
    // K * stride is whole float4s, the means 2 K d floats
    const float4* src = reinterpret_cast<const float4*>(tab);
    float4* dst = reinterpret_cast<float4*>(ts);
    const int nf = K * stride + 2 * K * d, n4 = nf / 4;
    for (int e = threadIdx.x; e < n4; e += blockDim.x) dst[e] = src[e];
    for (int e = 4 * n4 + threadIdx.x; e < nf; e += blockDim.x) ts[e] = tab[e];
  }
  __syncthreads();
  const double* mus = reinterpret_cast<const double*>(ts + (size_t)K * stride);
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const float u32 = 5.9604644775390625e-8f;   // 2^-24
  bool exact = *flag != 0;
  float tk[GMM_ZS_MAXK], ek[GMM_ZS_MAXK];
  float tmax = -INFINITY;
  if (!exact) {
    float y[DT];
#pragma unroll
    for (int j = 0; j < DT; ++j) y[j] = j < d ? Y[(size_t)n * d + j] : 0.0f;
    const int T = gmm_zs_row(d);
    for (int k = 0; k < K; ++k) {
      const float* L32 = ts + k * stride;
      const float* a = L32 + T;
      const double* mk = mus + (size_t)k * d;
      const float* sc = a + d;
      const float lpc = sc[0];
      if (lpc == -INFINITY) {   // weight 0: the term is exactly 0 here and in the reference
        tk[k] = -INFINITY;
        ek[k] = 0.0f;
        continue;
      }
      constexpr int DW = (DT + 3) / 4 * 4;   // whole float4s of row entries
      float w[DW];
      float W2 = 0.0f;
#pragma unroll
      for (int j = 0; j < DW; ++j) {
        w[j] = (j < DT && j < d) ? __double2float_rn(__dadd_rn((double)y[j < DT ? j : 0], -mk[j])) : 0.0f;
        W2 = __fmaf_rn(w[j], w[j], W2);
      }
      float e = 0.0f, t1 = 0.0f;
#pragma unroll
      for (int i = 0; i < DT; ++i) {
        if (i < d) {
          // row i in float4s; its padding is zero (exact zero products)
          const float4* Li = reinterpret_cast<const float4*>(L32 + gmm_zs_row(i));
          float s = 0.0f;
#pragma unroll
          for (int q = 0; q <= i / 4; ++q) {
            const float4 l = Li[q];
            s = __fmaf_rn(l.x, w[4 * q], s);
            s = __fmaf_rn(l.y, w[4 * q + 1], s);
            s = __fmaf_rn(l.z, w[4 * q + 2], s);
            s = __fmaf_rn(l.w, w[4 * q + 3], s);
          }
          e = __fmaf_rn(s, s, e);
          t1 = __fmaf_rn(fabsf(s), a[i], t1);
        }
      }
      // W >= ||w~|| (the sum of squares' rounding and the root's covered)
      const float W = __fsqrt_ru(__fmul_ru(W2, 1.0f + (float)(DT + 2) * u32));
      const float sd2 = __fmul_ru(__fmul_ru(W, W), sc[1]);
      const float E = __fmul_ru(__fadd_ru(__fadd_ru(__fmul_ru((float)(d + 1) * u32, e),
                                                    __fmul_ru(2.0f * u32, __fmul_ru(W, t1))),
                                          __fmul_ru(u32 * u32 * 1.01f, sd2)),
                                1.0f + 0x1p-16f);
      const float t = __fmaf_rn(-0.5f, e, lpc);
      const float eps = __fadd_ru(__fadd_ru(__fmul_ru(0.5f, E), __fmul_ru(u32, fabsf(lpc) + fabsf(t))),
                                  __fmul_ru(0x1p-40f, fabsf(lpc) + e + 1.0f));
      tk[k] = t;
      ek[k] = eps;
      if (!(t < INFINITY) || !(eps < INFINITY)) exact = true;   // non-finite
      tmax = fmaxf(tmax, t);
    }
    if (!(tmax >= -690.0f && tmax <= 690.0f)) exact = true;
  }
  int zk = -1;
  if (!exact) {
    // p~_k and an absolute bound A_k on |p~_k - p_k / p_max| (the exact value
    // lies in [exp(dt - x), exp(dt + x)], x = eps_k + u |dt| + 4u, binary32
    // exp within 4u); far components, whose bands are wide, weigh their width
    // by their tiny size
    float C[GMM_ZS_MAXK];
    float acc = 0.0f, err = 0.0f;
    for (int k = 0; k < K; ++k) {
      float p = 0.0f;
      if (tk[k] != -INFINITY) {
        const float dt = __fsub_rn(tk[k], tmax);
        p = expf(dt);
        const float x = __fadd_ru(__fadd_ru(ek[k], __fmul_ru(u32, fabsf(dt))), 4.0f * u32);
        const float up = __fmul_ru(expf(__fadd_ru(dt, x)), 1.0f + 8.0f * u32);
        const float dn = __fmul_rd(expf(__fsub_rd(dt, x)), 1.0f - 8.0f * u32);
        err = __fadd_ru(err, fmaxf(__fsub_ru(up, p), __fsub_ru(p, dn)));
      }
      acc = __fadd_rn(acc, p);
      C[k] = acc;
    }
    // band: the terms' errors, the running sums' and u * norm's roundings,
    // the comparisons' own roundings, the reference's running quotient sums
    const float Nt = C[K - 1];
    const float band = __fmul_ru(__fadd_ru(__fadd_ru(err, __fmul_ru((float)(K + 6) * u32, Nt)),
                                           __fmul_ru(0x1p-40f, Nt)), 1.0f + 0x1p-16f);
    Stream s = make_stream(seed, (uint32_t)n, iter, TAG_Z | (comp << 8));
    const double u = s.uniform();
    const float un = __fmul_rn(__double2float_rn(u), Nt);
    int i = 0;
    while (i < K - 1 && !(un < C[i])) ++i;
    const bool above_prev = i == 0 || __fadd_ru(C[i - 1], band) < __fsub_rd(un, band);
    const bool below_this = i == K - 1 || __fadd_ru(un, band) < __fsub_rd(C[i], band);
    if (above_prev && below_this && Nt >= 1.0f && band < INFINITY) zk = i;
  }
  if (zk >= 0) {
    z[n] = zk;
  } else {
    const int slot = atomicAdd(qn, 1);
    queue[slot] = n;
  }
}

// The reference's binary64 draw for the queued points, one CTA of K warps
// per point (K <= 32, d <= 32): warp k takes component k, lane i forms row
// i of Linv (y - mu_k) with gmm_z_kernel's operation order and lane 0 adds
// the squares in row order, all components side by side; thread 0 then
// makes the draw from the K densities.  CTAs take queued points in turn.
__global__ void __launch_bounds__(GMM_ZS_MAXK * 32)
gmm_zx_kernel(int d, int K, int shared_cov, const float* __restrict__ Y, const double* __restrict__ pis,
              const double* __restrict__ mu, const double* __restrict__ Linv, const double* __restrict__ hdet,
              const int* __restrict__ queue, const int* __restrict__ qn, int* __restrict__ z, uint64_t seed,
              uint32_t iter, uint32_t comp) {
  __shared__ double wsh[GMM_ZS_MAXK][32], ssh[GMM_ZS_MAXK][32], pmf[GMM_ZS_MAXK];
  const int lane = threadIdx.x & 31, k = threadIdx.x >> 5;
  const int nq = *qn;
  const double c = __dmul_rn(__dmul_rn(-0.5, (double)d), log(2.0 * 3.14159265358979323846264338327950288));
  const int kc = shared_cov ? 0 : k;
  const double* Lk = Linv + (size_t)kc * d * d;
  const double* mk = mu + (size_t)k * d;
  for (int q = blockIdx.x; q < nq; q += gridDim.x) {
    const int n = queue[q];
    if (lane < d) wsh[k][lane] = __dadd_rn((double)Y[(size_t)n * d + lane], -mk[lane]);
    __syncwarp();
    if (lane < d) {
      const double* Li = Lk + (size_t)lane * d;
      double s = 0.0;
#pragma unroll 4
      for (int jj = 0; jj <= lane; ++jj) s = __dadd_rn(s, __dmul_rn(Li[jj], wsh[k][jj]));
      ssh[k][lane] = s;
    }
    __syncwarp();
    if (lane == 0) {
      double expon = 0.0;
      for (int i = 0; i < d; ++i) expon = __dadd_rn(expon, __dmul_rn(ssh[k][i], ssh[k][i]));
      const double ll = __dadd_rn(__dadd_rn(c, -hdet[kc]), -__dmul_rn(0.5, expon));
      double prob = 1.0;
      prob = __dmul_rn(prob, pis[k]);
      prob = __dmul_rn(prob, exp(ll));
      pmf[k] = prob;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      Stream st = make_stream(seed, (uint32_t)n, iter, TAG_Z | (comp << 8));
      const double u = st.uniform();
      double norm = 0.0;
      for (int i = 0; i < K; ++i) norm = __dadd_rn(norm, pmf[i]);
      double acc = __ddiv_rn(pmf[0], norm);
      int zk = K - 1;
      for (int i = 1; i < K; ++i) {
        if (u < acc) { zk = i - 1; break; }
        acc = __dadd_rn(acc, __ddiv_rn(pmf[i], norm));
      }
      z[n] = zk;
    }
    __syncthreads();
  }
}

// ---- conjugate statistics ----------------------------------------------------
// CTA b accumulates points [b*chunk, (b+1)*chunk): counts, sum of y
// (want_sum) and the lower triangle of sum (y - mu_z)(y - mu_z)^T
// (want_obs; the reference's full-matrix update augur_mat_atm_inc_vtmt is
// symmetric elementwise).  The chunk is taken in sub-chunks of at most
// `sub` points: a sub-chunk's rows of Y are read with coalesced loads (all
// in flight at once) into shared memory, as binary32 rows when the sums are
// wanted and, for the scatter, centred once per point in binary64
// (c_i = y_i - mu_z,i, the value every scatter entry of the point uses);
// the points are sorted by component with a stable counting sort (warp 0,
// match_any ranks), and the components are walked one at a time: each
// thread owns fixed table entries and accumulates them in registers over
// the component's points in point order (a count is the component's number
// of points, the same double as adding 1.0 per point), adding the
// sub-chunk's sum to its partial.  Partials go to scratch [CTA][K][W] and
// gmm_stats_reduce_kernel adds them in CTA order (deterministic; the
// reference adds in point order).
constexpr int GMM_STAT_THREADS = 512;  // at d = 32 no thread owns more than two of the 529 scatter entries
constexpr int GMM_STAT_MAXE = 4;       // table entries per thread (W <= 4 * GMM_STAT_THREADS)
constexpr int GMM_STAT_SMEM = 96 * 1024;

// bytes of shared memory per point of a sub-chunk: label and rank, the
// binary32 row (sums), the centred binary64 row (scatter)
__host__ __device__ inline int gmm_stat_point_bytes(int d, int want_sum, int want_obs) {
  return 8 + (want_sum ? 4 * d : 0) + (want_obs ? 8 * d : 0);
}

__host__ __device__ inline int gmm_stat_sub(int d, int chunk, int want_sum, int want_obs) {
  const int fit = GMM_STAT_SMEM / gmm_stat_point_bytes(d, want_sum, want_obs);
  return chunk < fit ? chunk : fit;
}

__global__ void __launch_bounds__(GMM_STAT_THREADS)
gmm_stats_kernel(int N, int d, int K, const float* __restrict__ Y, const int* __restrict__ z,
                 const double* __restrict__ mu, int want_sum, int want_obs, int chunk,
                 double* __restrict__ part) {
  extern __shared__ double sdbl[];       // cs [sub][d] (double), then zs [sub], perm [sub], ys [sub][d] (float)
  __shared__ int koff[GMM_MAX_K + 1];
  const int sub = gmm_stat_sub(d, chunk, want_sum, want_obs);
  double* cs = sdbl;
  int* zs = reinterpret_cast<int*>(cs + (want_obs ? (size_t)sub * d : 0));
  int* perm = zs + sub;
  float* ys = reinterpret_cast<float*>(perm + sub);
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
    if (want_sum)
      for (int e = tid; e < m * d; e += blockDim.x) ys[e] = Y[(size_t)base * d + e];
    __syncthreads();
    if (want_obs) {
      // the centred rows, one binary64 subtraction per coordinate
      for (int e = tid; e < m * d; e += blockDim.x) {
        const int p = e / d, i = e - p * d;
        const int k = zs[p];
        cs[e] = k >= 0 ? __dadd_rn((double)Y[(size_t)base * d + e], -mu[(size_t)k * d + i]) : 0.0;
      }
    }
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
      const int p0 = koff[k], p1 = koff[k + 1];
#pragma unroll
      for (int q = 0; q < GMM_STAT_MAXE; ++q) {
        if (q >= ne) continue;
        double acc = 0.0;
        if (ekind[q] == 0) {
          acc = (double)(p1 - p0);                 // exactly the sum of p1 - p0 ones
        } else if (ekind[q] == 1) {
          const int i = ei[q];
          for (int p = p0; p < p1; ++p) acc = __dadd_rn(acc, (double)ys[perm[p] * d + i]);
        } else {
          const int i = ei[q], j = ej[q];
#pragma unroll 4
          for (int p = p0; p < p1; ++p) {
            const double* c = cs + perm[p] * d;
            acc = __dadd_rn(acc, __dmul_rn(c[i], c[j]));
          }
        }
        double* dst = part + ((size_t)blockIdx.x * K + k) * W + tid + q * blockDim.x;
        *dst = base == n0 ? acc : __dadd_rn(*dst, acc);
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
// reference's algorithm), spread over K * d CTAs.  Row i's sum of component
// k goes to chi[k * sk + i * si]: the diagonal of cov[k] (sk = d * d,
// si = d + 1), which gmm_conj_cov_kernel then reads and overwrites with the
// draw, or a [K][d] table of its own (sk = d, si = 1) when the draw runs
// beside the steps that still read cov.
__global__ void __launch_bounds__(GMM_THREADS)
gmm_bartlett_chi_kernel(int d, int df, const int* __restrict__ cnt, double* __restrict__ chi, int sk, int si,
                        uint64_t seed, uint32_t iter, uint32_t comp) {
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
  const double sum = block_sum_f64(local, red);
  if (threadIdx.x == 0) chi[(size_t)k * sk + (size_t)i * si] = sum;
}

// augur_invwishart_mvnormal_conj (augur_dist.c:751-757) and
// augur_invwishart_sample (:740-749) with bartlett_decomp (:722-738) for
// component k, one thread block, substream (k, iter, 9|comp<<8).  The
// Bartlett normals are drawn at the stream positions the reference's loop
// consumes them (row-major over the lower triangle; each diagonal
// chi-square of n - i normals follows its row's off-diagonal normals).  The
// chi-square sums of up to cnt + df squares come from
// gmm_bartlett_chi_kernel (chi[k * sk + i * si]), added in a fixed tree order
// instead of sequentially (a rounding-level difference); the d x d algebra
// runs on warp 0.
__global__ void __launch_bounds__(GMM_THREADS)
gmm_conj_cov_kernel(int d, int df, const double* __restrict__ scale0, const int* __restrict__ cnt,
                    const double* __restrict__ obs, const double* chi, int sk, int si, double* cov, uint64_t seed,
                    uint32_t iter, uint32_t comp) {
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
      A[e] = __dsqrt_rn(chi[(size_t)k * sk + (size_t)i * si]);
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

// Scratch of the screened draw: the component tables, the exact-path flag
// and queue length, the queue.
static inline size_t gmm_al256(size_t x) { return (x + 255) & ~(size_t)255; }
static inline size_t gmm_zs_smem(int d, int K) {
  return sizeof(float) * (size_t)K * gmm_zs_stride(d) + sizeof(double) * (size_t)K * d;
}
size_t gmm_zs_scratch(int N, int d, int K) { return gmm_al256(gmm_zs_smem(d, K)) + 256 + gmm_al256(sizeof(int) * (size_t)N); }
bool gmm_zs_fits(int d, int K) { return K <= GMM_ZS_MAXK && d <= 32 && gmm_zs_smem(d, K) <= 100 * 1024; }

template <int DT>
static int launch_zs_t(int N, int d, int K, const float* Y, const double* mu, const float* tab, const int* flag,
                       int* queue, int* qn, int* z, uint64_t seed, uint32_t iter, uint32_t comp, cudaStream_t st) {
  const size_t smem = gmm_zs_smem(d, K);
  AB_CUDA(cudaFuncSetAttribute(gmm_zs_kernel<DT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_zs_kernel<DT><<<ceil_div(N, GMM_ZS_THREADS), GMM_ZS_THREADS, smem, st>>>(N, d, K, Y, mu, tab, flag, queue, qn,
                                                                              z, seed, iter, comp);
  AB_LAUNCH_CHECK("gmm_zs_kernel");
  return AB_OK;
}

int launch_gmm_z_screened(int N, int d, int K, int shared, const float* Y, const double* pis, const double* mu,
                          const double* Linv, const double* hdet, int* z, uint64_t seed, uint32_t iter,
                          uint32_t comp, void* scratch, cudaStream_t st) {
  if (!gmm_zs_fits(d, K)) return launch_gmm_z(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, iter, comp, st);
  char* base = static_cast<char*>(scratch);
  float* tab = reinterpret_cast<float*>(base);
  int* ctl = reinterpret_cast<int*>(base + gmm_al256(gmm_zs_smem(d, K)));
  int* flag = ctl;
  int* qn = ctl + 1;
  int* queue = reinterpret_cast<int*>(reinterpret_cast<char*>(ctl) + 256);
  AB_CUDA(cudaMemsetAsync(ctl, 0, 2 * sizeof(int), st));
  gmm_zs_prep_kernel<<<K, 64, 0, st>>>(d, K, shared, pis, mu, Linv, hdet, tab, flag);
  AB_LAUNCH_CHECK("gmm_zs_prep_kernel");
  int rc;
  if (d <= 2) rc = launch_zs_t<2>(N, d, K, Y, mu, tab, flag, queue, qn, z, seed, iter, comp, st);
  else if (d <= 4) rc = launch_zs_t<4>(N, d, K, Y, mu, tab, flag, queue, qn, z, seed, iter, comp, st);
  else if (d <= 8) rc = launch_zs_t<8>(N, d, K, Y, mu, tab, flag, queue, qn, z, seed, iter, comp, st);
  else if (d <= 16) rc = launch_zs_t<16>(N, d, K, Y, mu, tab, flag, queue, qn, z, seed, iter, comp, st);
  else rc = launch_zs_t<32>(N, d, K, Y, mu, tab, flag, queue, qn, z, seed, iter, comp, st);
  if (rc) return rc;
  gmm_zx_kernel<<<592, 32 * K, 0, st>>>(d, K, shared, Y, pis, mu, Linv, hdet, queue, qn, z, seed, iter, comp);
  AB_LAUNCH_CHECK("gmm_zx_kernel");
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
  AB_REQUIRE(W <= GMM_STAT_MAXE * GMM_STAT_THREADS, AB_ERR_ARG, "gmm: d too large for the statistics pass");
  const int chunk = (N + GMM_STAT_CTAS - 1) / GMM_STAT_CTAS;
  const int nparts = (N + chunk - 1) / chunk;
  const int sub = gmm_stat_sub(d, chunk, want_sum, want_obs);
  const size_t smem = (size_t)gmm_stat_point_bytes(d, want_sum, want_obs) * (size_t)sub;
  AB_CUDA(cudaFuncSetAttribute(gmm_stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gmm_stats_kernel<<<nparts, GMM_STAT_THREADS, smem, st>>>(N, d, K, Y, z, mu, want_sum, want_obs, chunk, part);
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

// The Bartlett chi-square sums into chi (chi == nullptr: cov's diagonal).
int launch_gmm_bartlett(int K, int d, int df, const int* cnt, double* chi, double* cov, uint64_t seed,
                        uint32_t iter, uint32_t comp, cudaStream_t st) {
  if (chi != nullptr)
    gmm_bartlett_chi_kernel<<<K * d, GMM_THREADS, 0, st>>>(d, df, cnt, chi, d, 1, seed, iter, comp);
  else
    gmm_bartlett_chi_kernel<<<K * d, GMM_THREADS, 0, st>>>(d, df, cnt, cov, d * d, d + 1, seed, iter, comp);
  AB_LAUNCH_CHECK("gmm_bartlett_chi_kernel");
  return AB_OK;
}

// The inverse-Wishart draw from the chi-square sums in chi (chi == nullptr:
// cov's diagonal).
int launch_gmm_conj_cov_from(int K, int d, int df, const double* scale0, const int* cnt, const double* obs,
                             const double* chi, double* cov, uint64_t seed, uint32_t iter, uint32_t comp,
                             cudaStream_t st) {
  const size_t smem = sizeof(double) * 4 * (size_t)d * d;
  AB_CUDA(cudaFuncSetAttribute(gmm_conj_cov_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (chi != nullptr)
    gmm_conj_cov_kernel<<<K, GMM_THREADS, smem, st>>>(d, df, scale0, cnt, obs, chi, d, 1, cov, seed, iter, comp);
  else
    gmm_conj_cov_kernel<<<K, GMM_THREADS, smem, st>>>(d, df, scale0, cnt, obs, cov, d * d, d + 1, cov, seed, iter,
                                                      comp);
  AB_LAUNCH_CHECK("gmm_conj_cov_kernel");
  return AB_OK;
}

int launch_gmm_conj_cov(int K, int d, int df, const double* scale0, const int* cnt, const double* obs,
                        double* cov, uint64_t seed, uint32_t iter, uint32_t comp, cudaStream_t st) {
  int rc = launch_gmm_bartlett(K, d, df, cnt, nullptr, cov, seed, iter, comp, st);
  if (rc) return rc;
  return launch_gmm_conj_cov_from(K, d, df, scale0, cnt, obs, nullptr, cov, seed, iter, comp, st);
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

extern "C" size_t ab_gmm_z_scratch_bytes(int N, int d, int K) {
  if (N <= 0 || d <= 0 || K <= 0) return 0;
  return gmm_zs_scratch(N, d, K);
}

extern "C" size_t ab_gmm_z_queue_offset(int d, int K) {
  if (d <= 0 || K <= 0) return 0;
  return gmm_al256(gmm_zs_smem(d, K)) + sizeof(int);
}

extern "C" int ab_gmm_disc_z_screened(int N, int d, int K, int shared_cov, const float* Y, const double* pis,
                                      const double* mu, const double* Linv, const double* hdet, int* z,
                                      uint64_t seed, uint32_t iter, uint32_t comp, void* scratch, void* stream) {
  int rc = gmm_check(N, d, K);
  if (rc) return rc;
  AB_REQUIRE(Y && pis && mu && Linv && hdet && z && scratch, AB_ERR_ARG, "ab_gmm_disc_z_screened: null pointer");
  AB_REQUIRE((reinterpret_cast<uintptr_t>(scratch) & 255) == 0, AB_ERR_ARG,
             "ab_gmm_disc_z_screened: scratch must be 256-byte aligned");
  return launch_gmm_z_screened(N, d, K, shared_cov, Y, pis, mu, Linv, hdet, z, seed, iter, comp, scratch,
                               as_stream(stream));
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

extern "C" int ab_gmm_bartlett(int K, int d, int df, const int* cnt, double* chi, uint64_t seed, uint32_t iter,
                               uint32_t comp, void* stream) {
  AB_REQUIRE(K > 0 && K <= GMM_MAX_K && d > 0 && d <= GMM_MAX_D, AB_ERR_ARG, "ab_gmm_bartlett: bad sizes");
  AB_REQUIRE(df > 0 && df < 100000, AB_ERR_ARG, "ab_gmm_bartlett: bad degrees of freedom");
  AB_REQUIRE(cnt && chi, AB_ERR_ARG, "ab_gmm_bartlett: null pointer");
  return launch_gmm_bartlett(K, d, df, cnt, chi, nullptr, seed, iter, comp, as_stream(stream));
}

extern "C" int ab_gmm_conj_cov_chi(int K, int d, int df, const double* scale0, const int* cnt, const double* obs,
                                   const double* chi, double* cov, uint64_t seed, uint32_t iter, uint32_t comp,
                                   void* stream) {
  AB_REQUIRE(K > 0 && K <= GMM_MAX_K && d > 0 && d <= GMM_MAX_D, AB_ERR_ARG, "ab_gmm_conj_cov_chi: bad sizes");
  AB_REQUIRE(df > 0 && df < 100000, AB_ERR_ARG, "ab_gmm_conj_cov_chi: bad degrees of freedom");
  AB_REQUIRE(scale0 && cnt && obs && chi && cov, AB_ERR_ARG, "ab_gmm_conj_cov_chi: null pointer");
  return launch_gmm_conj_cov_from(K, d, df, scale0, cnt, obs, chi, cov, seed, iter, comp, as_stream(stream));
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
