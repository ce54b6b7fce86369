// LDA collapsed-free Gibbs sweep for the reference schedule
//   ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z]
// over the model of compiler/augur/test/lda.rv.
//
// Layout in HBM (all row-major):
//   w        int32 [T]      token ids, documents contiguous
//   doc_off  int32 [D+1]    CSR offsets of documents into w / z
//   z        int32 [T]      topic assignments
//   theta    f64   [D][K]   document-topic proportions
//   phiT     f64   [V][Kp]  topic-word proportions stored word-major, each
//                           row padded to Kp = round_up(K, 4) doubles so
//                           that a token's K values are one aligned segment
//   cnt_dk   int32 [D][K]   document-topic counts
//   cnt_kw   int32 [K][V]   topic-word counts
//
// One sweep is four kernels (theta runs concurrently with the phi pair):
//   lda_theta_kernel  theta[d] ~ Dir(alpha + cnt_dk[d])      (reads cnt_dk)
//   lda_phi_draw_kernel + lda_phi_norm_kernel
//                     phi[k]   ~ Dir(beta + cnt_kw[k])       (reads, then
//                     clears cnt_kw); one draw per thread, then a parallel
//                     normalisation pass
//   lda_zq_kernel     z ~ p(z | theta, phi), and the counts of the new z
//                     (cnt_dk rows written whole, cnt_kw incremented)
// The count statistics of the reference (conj_stat_*, rebuilt from zero each
// step, CgKern.hs:103-107) are a function of z alone, so they are produced
// by the z kernel of the previous sweep instead of by a separate pass.
//
// Bit-exactness: the z draw follows cbits/augur_dist.c:798-813 and
// CgDisc.hs:132-139 operation for operation in binary64 with no contraction
// (_rn intrinsics; this file is also compiled with -fmad=false), so given the
// same theta, phi and Philox uniforms the assignments and counts equal the
// reference's CPU sampler's bit for bit.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "dist.cuh"

namespace ab {

constexpr int LDA_THREADS = 256;
constexpr int LDA_MAX_K = 1024;
constexpr int LDA_PHI_MAX_B = 512;   // phi draw CTAs per topic whose partials are staged in shared memory

__device__ __forceinline__ uint32_t read_iter(const uint32_t* iter_dev, uint32_t iter_fixed) {
  return iter_dev ? *(volatile const uint32_t*)iter_dev : iter_fixed;
}

// ---------------------------------------------------------------------------
// theta[d][k] = g[d][k] / sum_k g[d][k],  g ~ Gamma(alpha_k + cnt[d][k], 1)
// (augur_dirichlet_categorical_conj, cbits/augur_dist.c:526-538).  The row
// sum is taken sequentially over k by one thread, as the reference does, so
// theta is bit-identical to the reference given identical gamma draws.
// Block: R = 256 / K rows (or one row looped when K > 256).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(LDA_THREADS, 4)
lda_theta_kernel(int D, int K, const double* __restrict__ alpha,
                 const int* __restrict__ cnt_dk, double* __restrict__ theta,
                 uint64_t seed, const uint32_t* iter_dev, uint32_t iter_fixed) {
  extern __shared__ double sg[];  // [rows_per_block][K] gamma draws, then [rows] sums
  const uint32_t iter = read_iter(iter_dev, iter_fixed);
  const int rows = K <= LDA_THREADS ? LDA_THREADS / K : 1;
  const int row0 = blockIdx.x * rows;
  double* sums = sg + rows * K;
  for (int e = threadIdx.x; e < rows * K; e += blockDim.x) {
    const int r = e / K, k = e - r * K;
    const int d = row0 + r;
    if (d < D) {
      const size_t idx = (size_t)d * K + k;
      Stream s = make_stream(seed, (uint32_t)idx, iter, TAG_THETA);
      sg[e] = gamma_draw(s, __dadd_rn(alpha[k], (double)cnt_dk[idx]), 1.0);
    }
  }
  __syncthreads();
  if (threadIdx.x < rows && row0 + (int)threadIdx.x < D) {
    double acc = 0.0;
    const double* g = sg + threadIdx.x * K;
    for (int k = 0; k < K; ++k) acc = __dadd_rn(acc, g[k]);
    sums[threadIdx.x] = acc;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < rows * K; e += blockDim.x) {
    const int r = e / K;
    const int d = row0 + r;
    if (d < D) theta[(size_t)row0 * K + e] = __ddiv_rn(sg[e], sums[r]);
  }
}

// ---------------------------------------------------------------------------
// phi[k][v] = g[k][v] / sum_v g[k][v], g ~ Gamma(beta_v + cnt[k][v], 1),
// stored word-major into phiT[v][k].  Two kernels:
//  lda_phi_draw_kernel  one gamma draw per thread over K * B CTAs (B CTAs of
//                       256 words per topic); writes g unnormalised into
//                       phiT, clears the counts it read and stores the CTA's
//                       fixed-order partial sum in scratch (partial[k][b]);
//                       the last CTA of a topic (atomic ticket) adds the B
//                       partials in CTA order into nrm[k];
//  lda_phi_norm_kernel  divides phiT by nrm, one 16-byte pair per thread.
// The sum is deterministic but not in the reference's sequential order, so
// phi matches the reference to rounding, not bitwise.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(LDA_THREADS, 4)
lda_phi_draw_kernel(int K, int V, int Kp, int B, const double* __restrict__ beta,
                    int* __restrict__ cnt_kw, double* __restrict__ phiT, int clear_counts,
                    double* __restrict__ partial, uint32_t* __restrict__ ticket,
                    double* __restrict__ nrm, uint64_t seed, const uint32_t* iter_dev,
                    uint32_t iter_fixed) {
  __shared__ double red[33];
  __shared__ double part_s[LDA_PHI_MAX_B];
  __shared__ int last;
  const uint32_t iter = read_iter(iter_dev, iter_fixed);
  const int k = blockIdx.x / B;
  const int b = blockIdx.x - k * B;
  const int v = b * LDA_THREADS + threadIdx.x;
  double g = 0.0;
  if (v < V) {
    const size_t idx = (size_t)k * V + v;
    const int c = cnt_kw[idx];
    if (clear_counts) cnt_kw[idx] = 0;
    Stream s = make_stream(seed, (uint32_t)idx, iter, TAG_PHI);
    g = gamma_draw(s, __dadd_rn(beta[v], (double)c), 1.0);
    phiT[(size_t)v * Kp + k] = g;
  }
  const double bsum = block_sum_f64(g, red);
  // The last CTA of topic k (atomic ticket) adds the topic's B partials in
  // CTA order and publishes the normaliser.  Its threads first load the B
  // partials together (one L2 round trip instead of B dependent ones); the
  // additions stay sequential, in CTA order.
  if (threadIdx.x == 0) {
    partial[(size_t)k * B + b] = bsum;
    __threadfence();
    last = atomicAdd(ticket + k, 1u) == (unsigned)(B - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    const double* pk = partial + (size_t)k * B;
    if (B <= LDA_PHI_MAX_B) {
      for (int i = threadIdx.x; i < B; i += blockDim.x) part_s[i] = __ldcg(pk + i);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      double acc = 0.0;
      for (int i = 0; i < B; ++i) acc = __dadd_rn(acc, B <= LDA_PHI_MAX_B ? part_s[i] : __ldcg(pk + i));
      nrm[k] = acc;
      ticket[k] = 0u;
    }
  }
}

// The same draw of phi for the sweep runner, with the rejection loops taken
// out of the draw kernel (three kernels instead of two):
//  lda_phi_try_kernel  one cell per thread, K * B CTAs of 256 words as
//                      lda_phi_draw_kernel: reads (and clears) the count,
//                      makes the cell's first Marsaglia-Tsang try
//                      (gamma_first_try) and stores the draws it decides; the
//                      undecided cells (about 5%) go to the CTA's queue, in
//                      thread order, with their counts; the CTA's block sum of
//                      its decided draws (zeros for the queued) goes to
//                      partial[cta];
//  lda_phi_fix_kernel  one warp per try CTA: completes the CTA's queued cells
//                      from their first try's normal and uniform
//                      (gamma_draw_resume), adds them to partial[cta] (each
//                      lane's draws in queue order, then a fixed butterfly),
//                      and the last warp of a topic (atomic ticket) adds the
//                      topic's B partials in CTA order into nrm[k];
//  lda_phi_norm_kernel as above.
// Every cell gets the draw gamma_draw gives it; the normaliser is a fixed-order
// (deterministic) sum.  No warp waits for another warp's rejection loop.
__global__ void __launch_bounds__(LDA_THREADS, 4)
lda_phi_try_kernel(int K, int V, int Kp, int B, const double* __restrict__ beta, int* __restrict__ cnt_kw,
                   double* __restrict__ phiT, int clear_counts, double* __restrict__ partial,
                   int2* __restrict__ queue, double2* __restrict__ queue_zu, int* __restrict__ qn,
                   uint64_t seed, const uint32_t* iter_dev, uint32_t iter_fixed) {
  __shared__ double red[33];
  __shared__ int wcount[LDA_THREADS / 32];
  const uint32_t iter = read_iter(iter_dev, iter_fixed);
  const int k = blockIdx.x / B;
  const int b = blockIdx.x - k * B;
  const int v = b * LDA_THREADS + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double g = 0.0, z1 = 0.0, u1 = 0.0;
  bool need = false;
  int c = 0;
  if (v < V) {
    const size_t idx = (size_t)k * V + v;
    c = cnt_kw[idx];
    if (clear_counts) cnt_kw[idx] = 0;
    Stream s = make_stream(seed, (uint32_t)idx, iter, TAG_PHI);
    if (gamma_first_try(s, __dadd_rn(beta[v], (double)c), 1.0, g, z1, u1)) {
      phiT[(size_t)v * Kp + k] = g;
    } else {
      need = true;
      g = 0.0;
    }
  }
  const unsigned bal = __ballot_sync(0xffffffffu, need);
  if (lane == 0) wcount[warp] = __popc(bal);
  const double bsum = block_sum_f64(g, red);     // its barriers also publish wcount
  if (need) {
    int base = 0;
    for (int i = 0; i < warp; ++i) base += wcount[i];
    const size_t slot = (size_t)blockIdx.x * LDA_THREADS + base + __popc(bal & ((1u << lane) - 1u));
    queue[slot] = make_int2(threadIdx.x, c);
    queue_zu[slot] = make_double2(z1, u1);
  }
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int i = 0; i < LDA_THREADS / 32; ++i) tot += wcount[i];
    qn[blockIdx.x] = tot;
    partial[blockIdx.x] = bsum;
  }
}

__global__ void __launch_bounds__(LDA_THREADS)
lda_phi_fix_kernel(int K, int V, int Kp, int B, const double* __restrict__ beta, double* __restrict__ phiT,
                   double* __restrict__ partial, const int2* __restrict__ queue,
                   const double2* __restrict__ queue_zu, const int* __restrict__ qn,
                   uint32_t* __restrict__ ticket, double* __restrict__ nrm, uint64_t seed,
                   const uint32_t* iter_dev, uint32_t iter_fixed) {
  const int lane = threadIdx.x & 31;
  const int cta = blockIdx.x * (LDA_THREADS / 32) + (threadIdx.x >> 5);
  if (cta >= K * B) return;                       // whole warps
  const uint32_t iter = read_iter(iter_dev, iter_fixed);
  const int k = cta / B;
  const int b = cta - k * B;
  const int n = qn[cta];
  double acc = 0.0;
  for (int i = lane; i < n; i += 32) {
    const int2 e = queue[(size_t)cta * LDA_THREADS + i];
    const double2 zu = queue_zu[(size_t)cta * LDA_THREADS + i];
    const int v = b * LDA_THREADS + e.x;
    const size_t idx = (size_t)k * V + v;
    Stream s = make_stream(seed, (uint32_t)idx, iter, TAG_PHI);
    s.pos = 2;                                  // after the try kernel's normal and uniform
    const double g = gamma_draw_resume(s, __dadd_rn(beta[v], (double)e.y), 1.0, zu.x, zu.y);
    phiT[(size_t)v * Kp + k] = g;
    acc = __dadd_rn(acc, g);
  }
  acc = warp_sum_f64(acc);
  int last = 0;
  if (lane == 0) {
    partial[cta] = __dadd_rn(partial[cta], acc);
    __threadfence();
    last = atomicAdd(ticket + k, 1u) == (unsigned)(B - 1);
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  // the topic's B partials in CTA order: the warp loads 32 at a time, lane 0 adds
  __threadfence();
  double tot = 0.0;
  for (int base = 0; base < B; base += 32) {
    const double x = base + lane < B ? __ldcg(partial + (size_t)k * B + base + lane) : 0.0;
    const int m = min(32, B - base);
    for (int j = 0; j < m; ++j) tot = __dadd_rn(tot, __shfl_sync(0xffffffffu, x, j));
  }
  if (lane == 0) {
    nrm[k] = tot;
    ticket[k] = 0u;
  }
}

// phiT [V][Kp] as V * Kp / 2 pairs of doubles; pair j holds topics 2j mod Kp
// and the next one.  Padding topics (k >= K) are left untouched (zero).
// When phi32 is given, the normalised values are also stored rounded to
// binary32 in phi32 [V][Kq] (the z kernel's screening copy; its padding
// columns are left untouched and must be zero).
__global__ void __launch_bounds__(LDA_THREADS)
lda_phi_norm_kernel(int K, int V, int Kp, const double* __restrict__ nrm_g,
                    double* __restrict__ phiT, float* __restrict__ phi32, int Kq) {
  extern __shared__ double nrm[];   // [K]
  for (int k = threadIdx.x; k < K; k += blockDim.x) nrm[k] = nrm_g[k];
  __syncthreads();
  const int half_kp = Kp >> 1;
  const size_t n2 = (size_t)V * half_kp;
  double2* p2 = reinterpret_cast<double2*>(phiT);
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += (size_t)gridDim.x * blockDim.x) {
    const int k = 2 * (int)(j % half_kp);
    if (k >= K) continue;
    double2 x = p2[j];
    x.x = __ddiv_rn(x.x, nrm[k]);
    if (k + 1 < K) x.y = __ddiv_rn(x.y, nrm[k + 1]);
    p2[j] = x;
    if (phi32 != nullptr) {
      const size_t v = j / half_kp;
      float2 f = make_float2(__double2float_rn(x.x), k + 1 < K ? __double2float_rn(x.y) : 0.0f);
      *reinterpret_cast<float2*>(phi32 + v * Kq + k) = f;
    }
  }
}

static inline int lda_phi_blocks(int V) { return (V + LDA_THREADS - 1) / LDA_THREADS; }

// Row stride (floats) of the binary32 screening copy of phi: a multiple of 8,
// so that each half row is whole 16-byte units.
static inline int lda_kq(int K) { return (K + 7) & ~7; }

// ---------------------------------------------------------------------------
// z[t] for every token of document d, K > 64 (one CTA per document; the
// staged kernel below takes K <= 64):
//   pmf_k  = (1 * theta[d][k]) * phi[k][w]                (CgDisc.hs:132-139)
//   norm   = sum_k pmf_k  (sequential)                    (augur_dist.c:800-803)
//   z      = first i with u < sum_{j<=i} pmf_j / norm      (:805-812)
// One lane per token, reading its phi row from global memory.  The norm pass
// records the running sum at 8 checkpoints; the reference's running quotient
// sum is replaced by a division-free test (comment in token_draw) evaluated
// first at the checkpoints and then inside the one block that contains the
// answer; only a u within rounding distance of a boundary runs the reference
// loop itself.  Products are recomputed where needed; they are the same
// binary64 values.
// Counts of the new z: the document's row of cnt_dk is accumulated in shared
// memory and stored whole; cnt_kw receives warp-aggregated atomic increments
// (lanes with the same (z, w) key elect one leader that adds the group size).
// ---------------------------------------------------------------------------
constexpr int LDA_Z_THREADS = 128;
constexpr int LDA_Z_CP = 8;            // checkpoints of the running sum

__device__ __forceinline__ int token_draw(int K, int half_kp, int nsuper, int R, int S,
                                          const double* __restrict__ th, const double* row,
                                          double u, double lo, double hi) {
  const double2* row2 = reinterpret_cast<const double2*>(row);
  const double2* th2 = reinterpret_cast<const double2*>(th);
  // Four interleaved partial sums shorten the floating-point dependency chain;
  // the fast test below tolerates any summation order of these nonnegative
  // products (its margin bounds the rounding of any order), and the exact
  // fallback recomputes the sequential sum.
  double cp[LDA_Z_CP];
#pragma unroll
  for (int i = 0; i < LDA_Z_CP; ++i) cp[i] = 0.0;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  for (int sc = 0; sc < nsuper; ++sc) {
    double2 f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int q = sc * 8 + i;
      f[i] = q < half_kp ? row2[q] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
      const int q = sc * 8 + i;
      const double2 g0 = th2[q], g1 = th2[q + 1];   // th is zero padded to KT
      a0 = __dadd_rn(a0, __dmul_rn(g0.x, f[i].x));
      a1 = __dadd_rn(a1, __dmul_rn(g0.y, f[i].y));
      a2 = __dadd_rn(a2, __dmul_rn(g1.x, f[i + 1].x));
      a3 = __dadd_rn(a3, __dmul_rn(g1.y, f[i + 1].y));
    }
    const int ci = sc / R;
    if (sc % R == R - 1 || sc == nsuper - 1) {
      const double c = __dadd_rn(__dadd_rn(a0, a1), __dadd_rn(a2, a3));
#pragma unroll
      for (int i = 0; i < LDA_Z_CP; ++i)
        if (i == ci) cp[i] = c;
    }
  }
  double norm = __dadd_rn(__dadd_rn(a0, a1), __dadd_rn(a2, a3));
#pragma unroll
  for (int i = 1; i < LDA_Z_CP; ++i)
    if (i > (nsuper - 1) / R) cp[i] = norm;
  // Division-free decision.  With c_j the running sum of the products,
  // u < acc_j (the reference's running sum of pmf_i / norm) holds when
  // u*norm < c_j (1 - m) and fails when u*norm > c_j (1 + m); m bounds the
  // rounding of both running sums, the quotients and the products
  // (|error| <= (2j + 3) 2^-53 relative, plus subnormal slack).  c_j is
  // nondecreasing, so a checkpoint with u*norm > c (1 + m) rules out its
  // whole block.  A u within m of a boundary takes the reference loop.
  bool exact = !(norm >= 1e-290 && norm <= 1.7976931348623157e308);
  int zk = K - 1;
  if (!exact) {
    const double un = __dmul_rn(u, norm);
    int blk = LDA_Z_CP - 1;
    double c = cp[LDA_Z_CP - 2];
#pragma unroll
    for (int i = LDA_Z_CP - 2; i >= 0; --i)
      if (un <= __dmul_rn(cp[i], hi)) { blk = i; c = i > 0 ? cp[i - 1] : 0.0; }
    const int j1 = min(K - 1, (blk + 1) * S);
    for (int j = blk * S; j < j1; ++j) {
      c = __dadd_rn(c, __dmul_rn(th[j], row[j]));
      if (un < __dmul_rn(c, lo)) { zk = j; break; }
      if (un <= __dmul_rn(c, hi)) { exact = true; break; }
    }
  }
  if (exact) {
    norm = 0.0;
    for (int k = 0; k < K; ++k) norm = __dadd_rn(norm, __dmul_rn(th[k], row[k]));
    double acc = __ddiv_rn(__dmul_rn(th[0], row[0]), norm);
    zk = K - 1;
    for (int i = 1; i < K; ++i) {
      if (u < acc) { zk = i - 1; break; }
      acc = __dadd_rn(acc, __ddiv_rn(__dmul_rn(th[i], row[i]), norm));
    }
  }
  return zk;
}

__global__ void __launch_bounds__(LDA_Z_THREADS, 4)
lda_z_kernel(int D, int K, int V, int Kp, const int* __restrict__ doc_off,
             const int* __restrict__ w, const double* __restrict__ theta,
             const double* __restrict__ phiT, int* __restrict__ z,
             int* __restrict__ cnt_dk, int* __restrict__ cnt_kw, uint64_t seed,
             uint32_t* iter_dev, uint32_t iter_fixed, uint32_t* done_ctr) {
  extern __shared__ double smem[];
  const int KT = 16 * ((K + 15) / 16);                  // theta padded to whole super-chunks
  double* th = smem;                                    // [KT] (zero padded)
  int* hist = reinterpret_cast<int*>(smem + KT);        // [K]
  const int half_kp = Kp / 2;
  const int lane = threadIdx.x & 31;
  const int d = blockIdx.x;
  const uint32_t iter = read_iter(iter_dev, iter_fixed);
  for (int k = threadIdx.x; k < KT; k += blockDim.x) {
    th[k] = k < K ? theta[(size_t)d * K + k] : 0.0;
    if (k < K) hist[k] = 0;
  }
  __syncthreads();
  const int t0 = doc_off[d], t1 = doc_off[d + 1];
  // Super-chunks of 16 doubles; a checkpoint block spans R of them.
  const int nsuper = (K + 15) / 16;
  const int R = (nsuper + LDA_Z_CP - 1) / LDA_Z_CP;
  const int S = 16 * R;                 // checkpoint block length in elements
  const double m = (6.0 * K + 32.0) * 1.1102230246251565e-16;
  const double lo = 1.0 - m, hi = 1.0 + m;
  const int nwarps = blockDim.x >> 5;
  for (int tb = t0 + (threadIdx.x >> 5) * 32; tb < t1; tb += nwarps * 32) {
    const int t = tb + lane;
    const bool active = t < t1;
    const int wt = active ? w[t] : 0;
    const double* row = phiT + (size_t)wt * Kp;
    int zk = 0;
    if (active) {
      Stream s = make_stream(seed, (uint32_t)t, iter, TAG_Z);
      const double u = s.uniform();
      zk = token_draw(K, half_kp, nsuper, R, S, th, row, u, lo, hi);
      z[t] = zk;
      atomicAdd(&hist[zk], 1);
    }
    if (cnt_kw != nullptr) {
      const unsigned mask = __ballot_sync(0xffffffffu, active);
      if (active) {
        const long long key = (long long)zk * V + wt;
        const unsigned peers = __match_any_sync(mask, key);
        const int leader = __ffs(peers) - 1;
        if (lane == leader) atomicAdd(cnt_kw + key, __popc(peers));
      }
    }
  }
  __syncthreads();
  if (cnt_dk != nullptr)
    for (int k = threadIdx.x; k < K; k += blockDim.x) cnt_dk[(size_t)d * K + k] = hist[k];
  // The last CTA to finish advances the device iteration counter, so a
  // captured sweep can be replayed without host updates.
  if (iter_dev != nullptr && done_ctr != nullptr) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned prev = atomicAdd(done_ctr, 1u);
      if (prev == (unsigned)(D - 1)) {
        *done_ctr = 0u;
        *iter_dev = iter + 1u;
        __threadfence();
      }
    }
  }
}

// The reference's draw itself (augur_unnorm_disc_samp, augur_dist.c:798-813,
// with pmf_k = (1 * theta_k) * phi_k of CgDisc.hs:132-139): a sequential norm,
// then the running sum of quotients.  Used where the division-free test of
// the grouped kernel cannot decide (u within rounding of a boundary, or a
// norm that is zero, subnormal, infinite or NaN).
__device__ __noinline__ int lda_reference_draw(int K, const double* __restrict__ th,
                                               const double* __restrict__ row, double u) {
  double norm = 0.0;
  for (int k = 0; k < K; ++k) norm = __dadd_rn(norm, __dmul_rn(th[k], row[k]));
  double acc = __ddiv_rn(__dmul_rn(th[0], row[0]), norm);
  int zk = K - 1;
  for (int i = 1; i < K; ++i) {
    if (u < acc) { zk = i - 1; break; }
    acc = __dadd_rn(acc, __ddiv_rn(__dmul_rn(th[i], row[i]), norm));
  }
  return zk;
}

// ---------------------------------------------------------------------------
// z[t] for every token of document d, K <= 64 (one CTA of 128 threads per
// document; NQ = Kp / 4 quads of topics, a compile-time constant).
// Each warp takes LDA_ZQ_ROWS (16) consecutive tokens, two lanes per token:
// lane j and lane j + 16 share token j, the first lane holding topics
// [0, 2 NQ) of its row and the second topics [2 NQ, 4 NQ).  The warp copies
// the chunk's phi rows into shared memory with asynchronous 16-byte copies,
// one row per copy instruction (a row is one contiguous segment, and all the
// chunk's rows are in flight at once); the row pitch is an odd number of
// 16-byte units so that the per-lane row reads that follow are bank-conflict
// free.  Each lane then makes one pass over its half row: p_k = theta_k *
// phi_k and the running sum of its half, written back over the row.  With A
// the first half's total, the running sum of the products is c_k for the
// first half and c_k = A + s_k for the second (s_k the second half's own
// running sum); norm = A + S (S the second half's total).  This groups the
// additions differently from the reference's sequential sum, by at most one
// rounding per term, which the margin below covers.
// The draw is the first k <= K - 2 with u < acc_k (acc_k the reference's
// running sum of p_j / norm); it is found without divisions by a binary
// search over the nondecreasing c_k (each lane in its half) for the first k
// with u norm <= c_k (1 + m), and is decided when also u norm < c_k (1 - m).
// m = (6K + 32) 2^-53 bounds the rounding of the products, sums (in either
// grouping) and quotients on both sides, so a decided draw equals the
// reference's; a u within m of a boundary (or a zero, subnormal, infinite or
// NaN norm) runs the reference's loop itself (lda_reference_draw).  theta
// and phi are probabilities (nonnegative), which keeps c_k monotone.
// Counts of the new z: the document's row of cnt_dk is accumulated in shared
// memory and stored whole; cnt_kw, when given, receives one atomic increment
// per token.
// ---------------------------------------------------------------------------
constexpr int LDA_ZQ_MAX_K = 64;

// Tokens per warp chunk: the 16 phi rows a warp stages at a time, two lanes
// per token.
constexpr int LDA_ZQ_ROWS = 16;

template <int NQ>
__global__ void __launch_bounds__(LDA_Z_THREADS, 8)
lda_zq_kernel(int D, int K, int V, const int* __restrict__ doc_off,
              const int* __restrict__ w, const double* __restrict__ theta,
              const double* __restrict__ phiT, int* __restrict__ z, int* __restrict__ cnt_dk, int* __restrict__ cnt_kw, uint64_t seed,
              uint32_t* iter_dev, uint32_t iter_fixed, uint32_t* done_ctr) {
  constexpr int KP = 4 * NQ;          // row length in doubles (= the phiT stride)
  constexpr int H2 = 2 * NQ;          // row length in 16-byte units
  constexpr int HK = 2 * NQ;          // topics per half row
  constexpr int P2 = H2 + 1;          // row pitch in 16-byte units (odd)
  // largest power of two <= HK: the search can return every count 0..HK
  constexpr int STEP0 = HK >= 32 ? 32 : (HK >= 16 ? 16 : (HK >= 8 ? 8 : (HK >= 4 ? 4 : (HK >= 2 ? 2 : 1))));
  extern __shared__ double2 smem2[];
  double2* th2 = smem2;                                        // [H2] theta, zero padded
  int* hist = reinterpret_cast<int*>(smem2 + H2);              // [KP]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = lane & 15, half = lane >> 4;
  double2* stage = smem2 + H2 + NQ + warp * LDA_ZQ_ROWS * P2;  // [LDA_ZQ_ROWS][P2] this warp's rows
  const int d = blockIdx.x;
  const uint32_t iter = read_iter(iter_dev, iter_fixed);
  double* th = reinterpret_cast<double*>(th2);
  for (int k = threadIdx.x; k < KP; k += blockDim.x) {
    th[k] = k < K ? theta[(size_t)d * K + k] : 0.0;
    hist[k] = 0;
  }
  __syncthreads();
  const int t0 = doc_off[d], t1 = doc_off[d + 1];
  const double m = (6.0 * K + 32.0) * 1.1102230246251565e-16;
  const double lo = 1.0 - m, hi = 1.0 + m;
  const double2* __restrict__ phi2 = reinterpret_cast<const double2*>(phiT);
  // topics of this lane's half that can be a draw's answer (k <= K - 2)
  const int n_half = min(max(K - 1 - half * HK, 0), HK);
  constexpr int STRIDE = (LDA_Z_THREADS / 32) * LDA_ZQ_ROWS;
  // word ids one chunk ahead: the load of the next chunk's ids is in flight
  // while this chunk computes, instead of preceding the next chunk's copies
  int w_next = (lane < LDA_ZQ_ROWS && t0 + warp * LDA_ZQ_ROWS + lane < t1) ? w[t0 + warp * LDA_ZQ_ROWS + lane] : 0;
  for (int tb = t0 + warp * LDA_ZQ_ROWS; tb < t1; tb += STRIDE) {
    const int t = tb + j;
    const bool active = t < t1;
    const int wt = w_next;
    w_next = (lane < LDA_ZQ_ROWS && tb + lane + STRIDE < t1) ? w[tb + lane + STRIDE] : 0;
    const int nrow = min(LDA_ZQ_ROWS, t1 - tb);
#pragma unroll
    for (int r = 0; r < LDA_ZQ_ROWS; ++r) {
      const int wr = __shfl_sync(0xffffffffu, wt, r);
      if (r < nrow && lane < H2) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(stage + r * P2 + lane);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst),
                     "l"(phi2 + (size_t)wr * H2 + lane) : "memory");
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    double u = 0.0;
    if (active && half == 0) {
      Stream s = make_stream(seed, (uint32_t)t, iter, TAG_Z);
      u = s.uniform();
    }
    u = __shfl_sync(0xffffffffu, u, j);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
    // running sum of this lane's half row, written back over it
    double2* row = stage + j * P2 + half * NQ;
    const double2* thh = th2 + half * NQ;
    double c = 0.0;
    if (active) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const double2 f = row[q], g = thh[q];
        const double c0 = __dadd_rn(c, __dmul_rn(g.x, f.x));
        c = __dadd_rn(c0, __dmul_rn(g.y, f.y));
        row[q] = make_double2(c0, c);
      }
    }
    const double A = __shfl_sync(0xffffffffu, c, j);          // first half's total
    const double S = __shfl_sync(0xffffffffu, c, j + 16);     // second half's total
    const double norm = __dadd_rn(A, S);                      // padding topics add exact zeros
    const double off = half ? A : 0.0;
    const double un = __dmul_rn(u, norm);
    const double* cs = reinterpret_cast<const double*>(row);
    // pos = number of k in this half's range with c_k (1 + m) < u norm (a prefix)
    int pos = 0;
#pragma unroll
    for (int step = STEP0; step >= 1; step >>= 1)
      if (pos + step <= n_half && __dmul_rn(__dadd_rn(off, cs[pos + step - 1]), hi) < un) pos += step;
    int cand = -1, dec = 0;
    if (pos < n_half) {
      cand = half * HK + pos;
      dec = un < __dmul_rn(__dadd_rn(off, cs[pos]), lo);
    }
    const int cand1 = __shfl_sync(0xffffffffu, cand, j + 16);
    const int dec1 = __shfl_sync(0xffffffffu, dec, j + 16);
    if (active && half == 0) {
      bool exact = !(norm >= 1e-290 && norm <= 1.7976931348623157e308);
      int zk = K - 1;
      if (!exact) {
        if (cand >= 0) { zk = cand; exact = !dec; }
        else if (cand1 >= 0) { zk = cand1; exact = !dec1; }
      }
      if (exact) zk = lda_reference_draw(K, th, phiT + (size_t)wt * KP, u);
      z[t] = zk;
      atomicAdd(&hist[zk], 1);
      // topic-word counts: one fire-and-forget atomic per token
      if (cnt_kw != nullptr) atomicAdd(cnt_kw + (size_t)zk * V + wt, 1);
    }
    __syncwarp();   // the stage is rewritten by the next chunk
  }
  __syncthreads();
  if (cnt_dk != nullptr)
    for (int k = threadIdx.x; k < K; k += blockDim.x) cnt_dk[(size_t)d * K + k] = hist[k];
  // The last CTA to finish advances the device iteration counter, so a
  // captured sweep can be replayed without host updates.
  if (iter_dev != nullptr && done_ctr != nullptr) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned prev = atomicAdd(done_ctr, 1u);
      if (prev == (unsigned)(D - 1)) {
        *done_ctr = 0u;
        *iter_dev = iter + 1u;
        __threadfence();
      }
    }
  }
}

template <int NQ>
static int launch_lda_zq(int D, int K, int V, const int* doc_off, const int* w, const double* theta,
                         const double* phiT, int* z, int* cnt_dk, int* cnt_kw, uint64_t seed,
                         uint32_t* iter_dev, uint32_t iter, uint32_t* done_ctr, cudaStream_t st) {
  const size_t smem = 16 * (size_t)(2 * NQ + NQ + (LDA_Z_THREADS / 32) * LDA_ZQ_ROWS * (2 * NQ + 1));
  AB_CUDA(cudaFuncSetAttribute(lda_zq_kernel<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  lda_zq_kernel<NQ><<<D, LDA_Z_THREADS, smem, st>>>(D, K, V, doc_off, w, theta, phiT, z, cnt_dk, cnt_kw, seed,
                                                    iter_dev, iter, done_ctr);
  AB_LAUNCH_CHECK("lda_zq_kernel");
  return AB_OK;
}

// ---------------------------------------------------------------------------
// The z draw screened in binary32 (K <= 64; NH = Kq / 8 16-byte units per
// half row, Kq = lda_kq(K)).  Same structure as lda_zq_kernel - one CTA per
// document, 16 tokens per warp chunk, two lanes per token (lane j: topics
// [0, 4 NH), lane j + 16: [4 NH, 8 NH)), the chunk's rows staged in shared
// memory by cp.async with an odd row pitch - but the staged rows are the
// binary32 copy phi32 = fl32(phi) (Kq floats: 224 bytes at K = 50 against 416
// for the binary64 rows) and the products and running sums are binary32.
//
// Why a decided draw is still the reference's: every theta_k, phi_k is
// rounded once to binary32 (relative error <= u = 2^-24), each product once
// more, and a running sum of nonnegative terms (grouped as two halves) adds
// at most (k + 1) u relative error, so each screened running sum c_k and the
// norm are within (K + 8) u of the exact sums C_k and N; u * norm adds 3 u.
// Gradual underflow adds at most 2^-149 per term, below 2^-60 u of a norm
// >= 2^-60.  The reference's running quotient sums acc_i are within 2^-50 of
// C_i / N.  So with m = (2K + 32) u: if c_j (1 + m) < u norm for all j < k the
// reference does not stop before k, and if also u norm < c_k (1 - m) it stops
// at k - the draw equals the reference's.  A u within the margin of a
// boundary (about 2 (2K + 32) u of the draws, 1e-5 at K = 50), or a norm
// outside [2^-60, FLT_MAX], runs the reference's binary64 loop on the binary64
// theta and phi rows (lda_reference_draw).  Counts as lda_zq_kernel.
// ---------------------------------------------------------------------------
template <int NH>
__global__ void __launch_bounds__(LDA_Z_THREADS, 10)
lda_zf_kernel(int D, int K, int V, int Kp, const int* __restrict__ doc_off,
              const int* __restrict__ w, const double* __restrict__ theta,
              const double* __restrict__ phiT, const float* __restrict__ phi32,
              int* __restrict__ z, int* __restrict__ cnt_dk, int* __restrict__ cnt_kw, uint64_t seed,
              uint32_t* iter_dev, uint32_t iter_fixed, uint32_t* done_ctr) {
  constexpr int KQ = 8 * NH;          // row length in floats (= the phi32 stride)
  constexpr int RU = 2 * NH;          // row length in 16-byte units
  constexpr int HK = 4 * NH;          // topics per half row
  constexpr int P2 = RU + 1;          // row pitch in 16-byte units (odd)
  // largest power of two <= HK: the search can return every count 0..HK
  constexpr int STEP0 = HK >= 32 ? 32 : (HK >= 16 ? 16 : (HK >= 8 ? 8 : 4));
  extern __shared__ float4 smem4[];
  float4* th4 = smem4;                                           // [RU] theta in binary32, zero padded
  int* hist = reinterpret_cast<int*>(smem4 + RU);                // [KQ]
  double* th64 = reinterpret_cast<double*>(smem4 + 2 * RU);      // [KQ] theta in binary64 (fallback)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = lane & 15, half = lane >> 4;
  float4* stage = smem4 + 2 * RU + 2 * RU + warp * LDA_ZQ_ROWS * P2;   // [LDA_ZQ_ROWS][P2]
  const int d = blockIdx.x;
  const uint32_t iter = read_iter(iter_dev, iter_fixed);
  float* th32 = reinterpret_cast<float*>(th4);
  for (int k = threadIdx.x; k < KQ; k += blockDim.x) {
    const double t = k < K ? theta[(size_t)d * K + k] : 0.0;
    th64[k] = t;
    th32[k] = __double2float_rn(t);
    hist[k] = 0;
  }
  __syncthreads();
  const int t0 = doc_off[d], t1 = doc_off[d + 1];
  const float m = (float)(2 * K + 32) * 5.9604644775390625e-8f;
  const float lo = 1.0f - m, hi = 1.0f + m;
  const float4* __restrict__ phi4 = reinterpret_cast<const float4*>(phi32);
  const int n_half = min(max(K - 1 - half * HK, 0), HK);
  constexpr int STRIDE = (LDA_Z_THREADS / 32) * LDA_ZQ_ROWS;
  int w_next = (lane < LDA_ZQ_ROWS && t0 + warp * LDA_ZQ_ROWS + lane < t1) ? w[t0 + warp * LDA_ZQ_ROWS + lane] : 0;
  for (int tb = t0 + warp * LDA_ZQ_ROWS; tb < t1; tb += STRIDE) {
    const int t = tb + j;
    const bool active = t < t1;
    const int wt = w_next;
    w_next = (lane < LDA_ZQ_ROWS && tb + lane + STRIDE < t1) ? w[tb + lane + STRIDE] : 0;
    const int nrow = min(LDA_ZQ_ROWS, t1 - tb);
    // two rows per copy instruction: lanes 0-15 row 2r, lanes 16-31 row 2r+1
#pragma unroll
    for (int r = 0; r < LDA_ZQ_ROWS / 2; ++r) {
      const int row = 2 * r + half;
      const int wr = __shfl_sync(0xffffffffu, wt, row);
      if (row < nrow && j < RU) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(stage + row * P2 + j);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst),
                     "l"(phi4 + (size_t)wr * RU + j) : "memory");
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    double u = 0.0;
    if (active && half == 0) {
      Stream s = make_stream(seed, (uint32_t)t, iter, TAG_Z);
      u = s.uniform();
    }
    u = __shfl_sync(0xffffffffu, u, j);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
    float4* row = stage + j * P2 + half * NH;
    const float4* thh = th4 + half * NH;
    float c = 0.0f;
    if (active) {
#pragma unroll
      for (int q = 0; q < NH; ++q) {
        const float4 f = row[q], g = thh[q];
        const float c0 = __fadd_rn(c, __fmul_rn(g.x, f.x));
        const float c1 = __fadd_rn(c0, __fmul_rn(g.y, f.y));
        const float c2 = __fadd_rn(c1, __fmul_rn(g.z, f.z));
        c = __fadd_rn(c2, __fmul_rn(g.w, f.w));
        row[q] = make_float4(c0, c1, c2, c);
      }
    }
    const float A = __shfl_sync(0xffffffffu, c, j);
    const float S = __shfl_sync(0xffffffffu, c, j + 16);
    const float norm = __fadd_rn(A, S);
    const float off = half ? A : 0.0f;
    const float un = __fmul_rn(__double2float_rn(u), norm);
    const float* cs = reinterpret_cast<const float*>(row);
    int pos = 0;
#pragma unroll
    for (int step = STEP0; step >= 1; step >>= 1)
      if (pos + step <= n_half && __fmul_rn(__fadd_rn(off, cs[pos + step - 1]), hi) < un) pos += step;
    int cand = -1, dec = 0;
    if (pos < n_half) {
      cand = half * HK + pos;
      dec = un < __fmul_rn(__fadd_rn(off, cs[pos]), lo);
    }
    const int cand1 = __shfl_sync(0xffffffffu, cand, j + 16);
    const int dec1 = __shfl_sync(0xffffffffu, dec, j + 16);
    if (active && half == 0) {
      bool exact = !(norm >= 8.673617379884035e-19f && norm <= 3.4028234663852886e38f);   // [2^-60, FLT_MAX]
      int zk = K - 1;
      if (!exact) {
        if (cand >= 0) { zk = cand; exact = !dec; }
        else if (cand1 >= 0) { zk = cand1; exact = !dec1; }
      }
      if (exact) zk = lda_reference_draw(K, th64, phiT + (size_t)wt * Kp, u);
      z[t] = zk;
      atomicAdd(&hist[zk], 1);
      if (cnt_kw != nullptr) atomicAdd(cnt_kw + (size_t)zk * V + wt, 1);
    }
    __syncwarp();   // the stage is rewritten by the next chunk
  }
  __syncthreads();
  if (cnt_dk != nullptr)
    for (int k = threadIdx.x; k < K; k += blockDim.x) cnt_dk[(size_t)d * K + k] = hist[k];
  if (iter_dev != nullptr && done_ctr != nullptr) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned prev = atomicAdd(done_ctr, 1u);
      if (prev == (unsigned)(D - 1)) {
        *done_ctr = 0u;
        *iter_dev = iter + 1u;
        __threadfence();
      }
    }
  }
}

template <int NH>
static int launch_lda_zf_t(int D, int K, int V, int Kp, const int* doc_off, const int* w, const double* theta,
                           const double* phiT, const float* phi32, int* z, int* cnt_dk, int* cnt_kw,
                           uint64_t seed, uint32_t* iter_dev, uint32_t iter, uint32_t* done_ctr,
                           cudaStream_t st) {
  // theta32 [2NH] + hist [2NH] + theta64 [2 * 2NH] + stages, in 16-byte units
  const size_t smem = 16 * (size_t)(2 * NH + 2 * NH + 2 * (2 * NH) + (LDA_Z_THREADS / 32) * LDA_ZQ_ROWS * (2 * NH + 1));
  AB_CUDA(cudaFuncSetAttribute(lda_zf_kernel<NH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  lda_zf_kernel<NH><<<D, LDA_Z_THREADS, smem, st>>>(D, K, V, Kp, doc_off, w, theta, phiT, phi32, z, cnt_dk,
                                                    cnt_kw, seed, iter_dev, iter, done_ctr);
  AB_LAUNCH_CHECK("lda_zf_kernel");
  return AB_OK;
}

int launch_lda_zf(int D, int K, int V, int Kp, const int* doc_off, const int* w, const double* theta,
                  const double* phiT, const float* phi32, int* z, int* cnt_dk, int* cnt_kw, uint64_t seed,
                  uint32_t* iter_dev, uint32_t iter, uint32_t* done_ctr, cudaStream_t st) {
  switch (lda_kq(K) / 8) {
#define AB_ZF(nh) \
  case nh: return launch_lda_zf_t<nh>(D, K, V, Kp, doc_off, w, theta, phiT, phi32, z, cnt_dk, cnt_kw, seed, iter_dev, iter, done_ctr, st);
    AB_ZF(1) AB_ZF(2) AB_ZF(3) AB_ZF(4) AB_ZF(5) AB_ZF(6) AB_ZF(7) AB_ZF(8)
#undef AB_ZF
    default: break;
  }
  return fail(AB_ERR_ARG, "lda: the binary32-screened z kernel takes K <= 64 (K=%d)", K);
}

// Count statistics of a given z (conj_stat_theta / conj_stat_phi of
// CgConj.hs:171-177): one CTA per document; cnt_kw must be zero on entry.
__global__ void __launch_bounds__(LDA_THREADS)
lda_count_kernel(int K, int V, const int* __restrict__ doc_off,
                 const int* __restrict__ w, const int* __restrict__ z,
                 int* __restrict__ cnt_dk, int* __restrict__ cnt_kw) {
  extern __shared__ int hist_s[];
  const int d = blockIdx.x;
  for (int k = threadIdx.x; k < K; k += blockDim.x) hist_s[k] = 0;
  __syncthreads();
  for (int t = doc_off[d] + threadIdx.x; t < doc_off[d + 1]; t += blockDim.x) {
    const int zk = z[t];
    atomicAdd(&hist_s[zk], 1);
    atomicAdd(cnt_kw + (size_t)zk * V + w[t], 1);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) cnt_dk[(size_t)d * K + k] = hist_s[k];
}

// ------------------------------- launchers ---------------------------------

static int check_lda_dims(int D, int K, int V) {
  AB_REQUIRE(D > 0 && K > 0 && V > 0, AB_ERR_ARG, "LDA sizes must be positive (D=%d K=%d V=%d)", D, K, V);
  AB_REQUIRE(K <= LDA_MAX_K, AB_ERR_ARG, "LDA supports K <= %d topics (got %d)", LDA_MAX_K, K);
  AB_REQUIRE((size_t)K * (size_t)V < (1ull << 32), AB_ERR_ARG, "K*V must be < 2^32");
  return AB_OK;
}

int launch_lda_theta(int D, int K, const double* alpha, const int* cnt_dk, double* theta,
                     uint64_t seed, const uint32_t* iter_dev, uint32_t iter, cudaStream_t st) {
  const int rows = K <= LDA_THREADS ? LDA_THREADS / K : 1;
  const size_t smem = sizeof(double) * ((size_t)rows * K + rows);
  lda_theta_kernel<<<ceil_div(D, rows), LDA_THREADS, smem, st>>>(D, K, alpha, cnt_dk, theta, seed,
                                                                 iter_dev, iter);
  AB_LAUNCH_CHECK("lda_theta_kernel");
  return AB_OK;
}

// scratch: [0,256) reserved for the sweep runner's counters, then
// ticket[K] (uint32, zero between calls), nrm[K], partial[K][B] (doubles),
// each region 256-byte aligned.
static inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t lda_phi_scratch(int K, int V) {
  return 256 + al256(4 * (size_t)K) + al256(8 * (size_t)K) + sizeof(double) * (size_t)K * lda_phi_blocks(V);
}

int launch_lda_phi(int K, int V, int Kp, const double* beta, int* cnt_kw, double* phiT, int clear,
                   void* scratch, uint64_t seed, const uint32_t* iter_dev, uint32_t iter,
                   cudaStream_t st, float* phi32 = nullptr) {
  const int B = lda_phi_blocks(V);
  char* base = static_cast<char*>(scratch) + 256;
  uint32_t* ticket = reinterpret_cast<uint32_t*>(base);
  double* nrm = reinterpret_cast<double*>(base + al256(4 * (size_t)K));
  double* partial = reinterpret_cast<double*>(base + al256(4 * (size_t)K) + al256(8 * (size_t)K));
  lda_phi_draw_kernel<<<K * B, LDA_THREADS, 0, st>>>(K, V, Kp, B, beta, cnt_kw, phiT, clear, partial,
                                                     ticket, nrm, seed, iter_dev, iter);
  AB_LAUNCH_CHECK("lda_phi_draw_kernel");
  const size_t n2 = (size_t)V * (Kp / 2);
  const unsigned nb = (unsigned)std::min<size_t>((n2 + LDA_THREADS - 1) / LDA_THREADS, 148u * 8u);
  lda_phi_norm_kernel<<<nb, LDA_THREADS, sizeof(double) * K, st>>>(K, V, Kp, nrm, phiT, phi32,
                                                                    lda_kq(K));
  AB_LAUNCH_CHECK("lda_phi_norm_kernel");
  return AB_OK;
}

int launch_lda_z(int D, int K, int V, int Kp, const int* doc_off, const int* w, const double* theta,
                 const double* phiT, int* z, int* cnt_dk, int* cnt_kw, uint64_t seed,
                 uint32_t* iter_dev, uint32_t iter, uint32_t* done_ctr, cudaStream_t st) {
#define AB_ZQ(nq)                                                                                      \
  case nq:                                                                                             \
    return launch_lda_zq<nq>(D, K, V, doc_off, w, theta, phiT, z, cnt_dk, cnt_kw, seed, iter_dev, iter, \
                             done_ctr, st);
  if (K <= LDA_ZQ_MAX_K) {
    switch (Kp / 4) {
      AB_ZQ(1) AB_ZQ(2) AB_ZQ(3) AB_ZQ(4) AB_ZQ(5) AB_ZQ(6) AB_ZQ(7) AB_ZQ(8)
      AB_ZQ(9) AB_ZQ(10) AB_ZQ(11) AB_ZQ(12) AB_ZQ(13) AB_ZQ(14) AB_ZQ(15) AB_ZQ(16)
      default: break;
    }
    return fail(AB_ERR_STATE, "lda: no z kernel for Kp=%d", Kp);
  }
#undef AB_ZQ
  // theta [KT] doubles, then hist [K] ints
  const size_t KT = 16 * (size_t)((K + 15) / 16);
  const size_t smem = sizeof(double) * KT + sizeof(int) * (size_t)K;
  lda_z_kernel<<<D, LDA_Z_THREADS, smem, st>>>(D, K, V, Kp, doc_off, w, theta, phiT, z, cnt_dk, cnt_kw,
                                               seed, iter_dev, iter, done_ctr);
  AB_LAUNCH_CHECK("lda_z_kernel");
  return AB_OK;
}

int launch_lda_count(int D, int K, int V, const int* doc_off, const int* w, const int* z,
                     int* cnt_dk, int* cnt_kw, cudaStream_t st) {
  AB_CUDA(cudaMemsetAsync(cnt_kw, 0, sizeof(int) * (size_t)K * V, st));
  lda_count_kernel<<<D, LDA_THREADS, sizeof(int) * K, st>>>(K, V, doc_off, w, z, cnt_dk, cnt_kw);
  AB_LAUNCH_CHECK("lda_count_kernel");
  return AB_OK;
}

static inline int lda_kp(int K) { return (K + 3) & ~3; }

}  // namespace ab

using namespace ab;

// ------------------------------- C ABI -------------------------------------

extern "C" int ab_lda_phi_stride(int K) { return lda_kp(K); }

extern "C" int ab_lda_count(int D, int K, int V, const int* doc_off, const int* w, const int* z,
                            int* cnt_dk, int* cnt_kw, void* stream) {
  int rc = check_lda_dims(D, K, V);
  if (rc) return rc;
  AB_REQUIRE(doc_off && w && z && cnt_dk && cnt_kw, AB_ERR_ARG, "ab_lda_count: null pointer");
  return launch_lda_count(D, K, V, doc_off, w, z, cnt_dk, cnt_kw, as_stream(stream));
}

extern "C" int ab_lda_conj_theta(int D, int K, const double* alpha, const int* cnt_dk, double* theta,
                                 uint64_t seed, uint32_t iter, void* stream) {
  AB_REQUIRE(D > 0 && K > 0 && K <= LDA_MAX_K, AB_ERR_ARG, "ab_lda_conj_theta: bad sizes D=%d K=%d", D, K);
  AB_REQUIRE(alpha && cnt_dk && theta, AB_ERR_ARG, "ab_lda_conj_theta: null pointer");
  return launch_lda_theta(D, K, alpha, cnt_dk, theta, seed, nullptr, iter, as_stream(stream));
}

extern "C" size_t ab_lda_phi_scratch_bytes(int K, int V) {
  return (K > 0 && V > 0) ? lda_phi_scratch(K, V) : 0;
}

extern "C" int ab_lda_conj_phi(int K, int V, const double* beta, int* cnt_kw, double* phiT,
                               int clear_counts, uint64_t seed, uint32_t iter, void* scratch,
                               void* stream) {
  int rc = check_lda_dims(1, K, V);
  if (rc) return rc;
  AB_REQUIRE(beta && cnt_kw && phiT && scratch, AB_ERR_ARG, "ab_lda_conj_phi: null pointer");
  cudaStream_t st = as_stream(stream);
  AB_CUDA(cudaMemsetAsync(static_cast<char*>(scratch) + 256, 0, 4 * (size_t)K, st));
  return launch_lda_phi(K, V, lda_kp(K), beta, cnt_kw, phiT, clear_counts, scratch, seed, nullptr,
                        iter, st);
}

extern "C" int ab_lda_disc_z(int D, int K, int V, const int* doc_off, const int* w,
                             const double* theta, const double* phiT, int* z, int* cnt_dk,
                             int* cnt_kw, uint64_t seed, uint32_t iter, void* stream) {
  int rc = check_lda_dims(D, K, V);
  if (rc) return rc;
  AB_REQUIRE(doc_off && w && theta && phiT && z, AB_ERR_ARG, "ab_lda_disc_z: null pointer");
  AB_REQUIRE((reinterpret_cast<uintptr_t>(phiT) & 15) == 0, AB_ERR_ARG, "ab_lda_disc_z: phiT must be 16-byte aligned");
  AB_REQUIRE((cnt_dk == nullptr) == (cnt_kw == nullptr), AB_ERR_ARG,
             "ab_lda_disc_z: pass both count tables or neither");
  return launch_lda_z(D, K, V, lda_kp(K), doc_off, w, theta, phiT, z, cnt_dk, cnt_kw, seed, nullptr, iter,
                      nullptr, as_stream(stream));
}

extern "C" int ab_lda_phi32_stride(int K) { return lda_kq(K); }

extern "C" int ab_lda_disc_z_f32(int D, int K, int V, const int* doc_off, const int* w, const double* theta,
                                 const double* phiT, const float* phi32, int* z, int* cnt_dk, int* cnt_kw,
                                 uint64_t seed, uint32_t iter, void* stream) {
  int rc = check_lda_dims(D, K, V);
  if (rc) return rc;
  AB_REQUIRE(K <= LDA_ZQ_MAX_K, AB_ERR_ARG, "ab_lda_disc_z_f32: K <= %d (got %d)", LDA_ZQ_MAX_K, K);
  AB_REQUIRE(doc_off && w && theta && phiT && phi32 && z, AB_ERR_ARG, "ab_lda_disc_z_f32: null pointer");
  AB_REQUIRE((reinterpret_cast<uintptr_t>(phi32) & 15) == 0, AB_ERR_ARG,
             "ab_lda_disc_z_f32: phi32 must be 16-byte aligned");
  AB_REQUIRE((cnt_dk == nullptr) == (cnt_kw == nullptr), AB_ERR_ARG,
             "ab_lda_disc_z_f32: pass both count tables or neither");
  return launch_lda_zf(D, K, V, lda_kp(K), doc_off, w, theta, phiT, phi32, z, cnt_dk, cnt_kw, seed, nullptr, iter,
                       nullptr, as_stream(stream));
}

// ---- variant of ab_lda_conj_phi that allocates nothing ----------------------
// Some callers cannot call cudaMalloc: a host framework that owns all device
// memory through its own pool and cannot hand out a raw scratch buffer, or a
// plugin that must not allocate while it runs.  For them the phi draw takes
// its scratch (per-CTA partial sums, per-topic normalisers and completion
// tickets) from this file-scope device array instead of a caller buffer.
// Every GPU that loads the library holds the array until the process exits.
constexpr size_t LDA_NOALLOC_SCRATCH_BYTES = 1u << 20;   // 1 MiB
static __device__ __align__(256) unsigned char g_lda_phi_scratch[LDA_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};   // device address of the array, per device ordinal
}  // namespace

extern "C" int ab_lda_conj_phi_noalloc(int K, int V, const double* beta, int* cnt_kw, double* phiT,
                                       int clear_counts, uint64_t seed, uint32_t iter, void* stream) {
  int rc = check_lda_dims(1, K, V);
  if (rc) return rc;
  AB_REQUIRE(beta && cnt_kw && phiT, AB_ERR_ARG, "ab_lda_conj_phi_noalloc: null pointer");
  const size_t need = lda_phi_scratch(K, V);
  AB_REQUIRE(need <= LDA_NOALLOC_SCRATCH_BYTES, AB_ERR_ARG,
             "ab_lda_conj_phi_noalloc: K=%d, V=%d need %zu bytes of scratch, above the built-in %zu; "
             "use ab_lda_conj_phi with a caller buffer",
             K, V, need, (size_t)LDA_NOALLOC_SCRATCH_BYTES);
  int dev = 0;
  AB_CUDA(cudaGetDevice(&dev));
  AB_REQUIRE(dev >= 0 && dev < 64, AB_ERR_ARG, "ab_lda_conj_phi_noalloc: device ordinal %d >= 64", dev);
  void* scratch = nullptr;
  {
    // First call on a device: look up the device address of the array (the
    // host-side name is only a stand-in and must never reach a kernel).
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
      void* p = nullptr;
      AB_CUDA(cudaGetSymbolAddress(&p, g_lda_phi_scratch));
      g_noalloc_ptr[dev] = p;
    }
    scratch = g_noalloc_ptr[dev];
  }
  cudaStream_t st = as_stream(stream);
  // the completion tickets must start at zero
  AB_CUDA(cudaMemsetAsync(static_cast<char*>(scratch) + 256, 0, 4 * (size_t)K, st));
  return launch_lda_phi(K, V, lda_kp(K), beta, cnt_kw, phiT, clear_counts, scratch, seed, nullptr, iter, st);
}

// ---- sweep runner with a captured CUDA graph -------------------------------

struct ab_lda {
  ab_lda_desc d;
  int Kp;
  cudaGraphExec_t exec = nullptr;
  int graph_sweeps = 0;
  cudaStream_t s_main = nullptr, s_side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

// Sweep scratch: the phi draw's scratch, whose first 256 bytes hold the
// runner's iteration and completion counters, then (K <= 64) the binary32
// screening copy of phi, phi32 f32 [V][Kq], zero padded, ...
static inline size_t lda_phi32_offset(int K, int V) { return al256(lda_phi_scratch(K, V)); }
static inline size_t lda_queue_offset(int K, int V) {
  return lda_phi32_offset(K, V) + al256(K <= LDA_ZQ_MAX_K ? sizeof(float) * (size_t)V * lda_kq(K) : 0);
}
// ... then the try kernel's queues: cells int2 [K * B][256], their first
// tries' (normal, uniform) double2 [K * B][256], and lengths int [K * B]
static inline size_t lda_sweep_scratch(int K, int V) {
  const size_t nb = (size_t)K * lda_phi_blocks(V);
  return lda_queue_offset(K, V) + (sizeof(int2) + sizeof(double2)) * nb * LDA_THREADS + sizeof(int) * nb;
}

// The sweep's phi draw: try (part 0), then fix and normalise (part 1)
// (lda_phi_try_kernel).
static int launch_lda_phi_sweep(int part, int K, int V, int Kp, const double* beta, int* cnt_kw, double* phiT,
                                void* scratch, float* phi32, uint64_t seed, const uint32_t* iter_dev,
                                cudaStream_t st) {
  const int B = lda_phi_blocks(V);
  char* base = static_cast<char*>(scratch) + 256;
  uint32_t* ticket = reinterpret_cast<uint32_t*>(base);
  double* nrm = reinterpret_cast<double*>(base + al256(4 * (size_t)K));
  double* partial = reinterpret_cast<double*>(base + al256(4 * (size_t)K) + al256(8 * (size_t)K));
  double2* queue_zu = reinterpret_cast<double2*>(static_cast<char*>(scratch) + lda_queue_offset(K, V));
  int2* queue = reinterpret_cast<int2*>(queue_zu + (size_t)K * B * LDA_THREADS);
  int* qn = reinterpret_cast<int*>(queue + (size_t)K * B * LDA_THREADS);
  if (part == 0) {
    lda_phi_try_kernel<<<K * B, LDA_THREADS, 0, st>>>(K, V, Kp, B, beta, cnt_kw, phiT, 1, partial, queue,
                                                      queue_zu, qn, seed, iter_dev, 0);
    AB_LAUNCH_CHECK("lda_phi_try_kernel");
    return AB_OK;
  }
  const int warps_per_cta = LDA_THREADS / 32;
  lda_phi_fix_kernel<<<ceil_div((size_t)K * B, warps_per_cta), LDA_THREADS, 0, st>>>(
      K, V, Kp, B, beta, phiT, partial, queue, queue_zu, qn, ticket, nrm, seed, iter_dev, 0);
  AB_LAUNCH_CHECK("lda_phi_fix_kernel");
  const size_t n2 = (size_t)V * (Kp / 2);
  const unsigned nb = (unsigned)std::min<size_t>((n2 + LDA_THREADS - 1) / LDA_THREADS, 148u * 8u);
  lda_phi_norm_kernel<<<nb, LDA_THREADS, sizeof(double) * K, st>>>(K, V, Kp, nrm, phiT, phi32, lda_kq(K));
  AB_LAUNCH_CHECK("lda_phi_norm_kernel");
  return AB_OK;
}

static int lda_enqueue_sweep(ab_lda* h, cudaStream_t main, cudaStream_t side) {
  const ab_lda_desc& d = h->d;
  uint32_t* iter_dev = reinterpret_cast<uint32_t*>(d.scratch);
  uint32_t* done = iter_dev + 1;
  float* phi32 = d.K <= LDA_ZQ_MAX_K
                     ? reinterpret_cast<float*>(static_cast<char*>(d.scratch) + lda_phi32_offset(d.K, d.V))
                     : nullptr;
  if (phi32 != nullptr) {
    // phi's first tries use the whole GPU; the theta draw then runs beside the
    // phi fix-up and normalisation, which leave most SMs idle
    int rc = launch_lda_phi_sweep(0, d.K, d.V, h->Kp, d.beta, d.cnt_kw, d.phiT, d.scratch, phi32, d.seed,
                                  iter_dev, main);
    if (rc) return rc;
    AB_CUDA(cudaEventRecord(h->fork, main));
    AB_CUDA(cudaStreamWaitEvent(side, h->fork, 0));
    rc = launch_lda_theta(d.D, d.K, d.alpha, d.cnt_dk, d.theta, d.seed, iter_dev, 0, side);
    if (rc) return rc;
    AB_CUDA(cudaEventRecord(h->join, side));
    rc = launch_lda_phi_sweep(1, d.K, d.V, h->Kp, d.beta, d.cnt_kw, d.phiT, d.scratch, phi32, d.seed, iter_dev,
                              main);
    if (rc) return rc;
    AB_CUDA(cudaStreamWaitEvent(main, h->join, 0));
    return launch_lda_zf(d.D, d.K, d.V, h->Kp, d.doc_off, d.w, d.theta, d.phiT, phi32, d.z, d.cnt_dk,
                         d.cnt_kw, d.seed, iter_dev, 0, done, main);
  }
  // K > 64: theta beside the two-kernel phi draw, then the binary64 z kernel
  AB_CUDA(cudaEventRecord(h->fork, main));
  AB_CUDA(cudaStreamWaitEvent(side, h->fork, 0));
  int rc = launch_lda_theta(d.D, d.K, d.alpha, d.cnt_dk, d.theta, d.seed, iter_dev, 0, main);
  if (rc) return rc;
  rc = launch_lda_phi(d.K, d.V, h->Kp, d.beta, d.cnt_kw, d.phiT, 1, d.scratch, d.seed, iter_dev, 0, side);
  if (rc) return rc;
  AB_CUDA(cudaEventRecord(h->join, side));
  AB_CUDA(cudaStreamWaitEvent(main, h->join, 0));
  return launch_lda_z(d.D, d.K, d.V, h->Kp, d.doc_off, d.w, d.theta, d.phiT, d.z, d.cnt_dk, d.cnt_kw,
                      d.seed, iter_dev, 0, done, main);
}

extern "C" size_t ab_lda_scratch_bytes(int K, int V) {
  return (K > 0 && V > 0) ? lda_sweep_scratch(K, V) : 0;
}

extern "C" int ab_lda_create(const ab_lda_desc* desc, ab_lda** out) {
  AB_REQUIRE(desc && out, AB_ERR_ARG, "ab_lda_create: null argument");
  int rc = check_lda_dims(desc->D, desc->K, desc->V);
  if (rc) return rc;
  AB_REQUIRE(desc->doc_off && desc->w && desc->z && desc->theta && desc->phiT && desc->alpha &&
                 desc->beta && desc->cnt_dk && desc->cnt_kw && desc->scratch,
             AB_ERR_ARG, "ab_lda_create: every device pointer of the descriptor is required");
  AB_REQUIRE((reinterpret_cast<uintptr_t>(desc->phiT) & 15) == 0, AB_ERR_ARG, "ab_lda_create: phiT must be 16-byte aligned");
  ab_lda* h = new ab_lda();
  h->d = *desc;
  h->Kp = lda_kp(desc->K);
  cudaError_t e = cudaStreamCreateWithFlags(&h->s_main, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->s_side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    ab_lda_destroy(h);
    return cuda_status(e, "ab_lda_create");
  }
  *out = h;
  return AB_OK;
}

extern "C" int ab_lda_init_state(ab_lda* h, uint32_t iter, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_lda_init_state: null handle");
  const ab_lda_desc& d = h->d;
  cudaStream_t st = as_stream(stream);
  AB_CUDA(cudaMemsetAsync(d.scratch, 0, lda_sweep_scratch(d.K, d.V), st));
  AB_CUDA(cudaMemcpyAsync(d.scratch, &iter, sizeof(iter), cudaMemcpyHostToDevice, st));
  return launch_lda_count(d.D, d.K, d.V, d.doc_off, d.w, d.z, d.cnt_dk, d.cnt_kw, st);
}

extern "C" int ab_lda_run(ab_lda* h, int n_sweeps, int use_graph, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_lda_run: null handle");
  AB_REQUIRE(n_sweeps >= 0, AB_ERR_ARG, "ab_lda_run: n_sweeps < 0");
  cudaStream_t st = as_stream(stream);
  if (!use_graph) {
    for (int s = 0; s < n_sweeps; ++s) {
      int rc = lda_enqueue_sweep(h, st, h->s_side);
      if (rc) return rc;
    }
    return AB_OK;
  }
  if (h->exec == nullptr) {
    cudaGraph_t g = nullptr;
    AB_CUDA(cudaStreamBeginCapture(h->s_main, cudaStreamCaptureModeThreadLocal));
    int rc = lda_enqueue_sweep(h, h->s_main, h->s_side);
    cudaError_t e = cudaStreamEndCapture(h->s_main, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    AB_CUDA(e);
    e = cudaGraphInstantiate(&h->exec, g, 0);
    cudaGraphDestroy(g);
    AB_CUDA(e);
  }
  for (int s = 0; s < n_sweeps; ++s) AB_CUDA(cudaGraphLaunch(h->exec, st));
  return AB_OK;
}

extern "C" int ab_lda_destroy(ab_lda* h) {
  if (!h) return AB_OK;
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->fork) cudaEventDestroy(h->fork);
  if (h->join) cudaEventDestroy(h->join);
  if (h->s_main) cudaStreamDestroy(h->s_main);
  if (h->s_side) cudaStreamDestroy(h->s_side);
  delete h;
  return AB_OK;
}
