// Hierarchical logistic regression: log-density and gradient over the data,
// and the HMC / NUTS / MWG transitions that consume them.
//
// Model (compiler/augur/test/hlr.rv, and its InvGamma-variance variant
// without the bias):
//   v ~ Exponential(lam) | InvGamma(a0, s0);  b ~ Normal(0, v)  (optional)
//   theta[k] ~ Normal(0, v);  y[n] ~ Bernoulli(sigmoid(theta . x[n] + b))
// Parameters of a chain are one binary64 vector par = [theta[0..D-1], b, v];
// a block (the unit an HMC / NUTS kernel moves) is a list of indices into par
// in the schedule's order.
//
// Data layout in HBM: X row-major [N][ldx] (f32 or bf16), y int32 [N],
// par f64 [C][D+2].
//
// Engine: one CTA per chain runs whole iterations of the schedule on chip
// (hlr_chain_kernel).  A data pass computes, at the chain's current theta
// and b, ll_data = sum_n log Bern(y_n | sigmoid(t_n)) and its gradient
//   d/dtheta_k = sum_n r_n x_nk,  d/db = sum_n r_n,  r_n = y_n - sigmoid(t_n)
// in FP32 per row (numerically stable logistic terms), with Kahan-compensated
// per-thread sums and fixed-order FP64 block reductions, so the result is
// deterministic.  Priors, momenta, energies and the accept tests are binary64
// in the reference's operation order (cbits/augur_dist.c, augur_mcmclib.h).
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"
#include "philox.cuh"

namespace ab {

constexpr int HLR_THREADS = 256;
constexpr int HLR_CHUNK = 1024;          // rows per data-pass chunk (r buffer)
constexpr int HLR_MAX_COLS = 4;          // columns per thread in the gradient pass
constexpr int HLR_MAX_D = HLR_THREADS * HLR_MAX_COLS - 1;
constexpr int HLR_STK = 16;              // NUTS stack entries (cbits/augur_blkstk.h:26)
constexpr int HLR_MAX_COMPS = 8;

enum { COMP_HMC = 0, COMP_NUTS = 1, COMP_MWG = 2, COMP_RSLICE = 3 };

struct HlrModelDev {
  int N, D, ldx, has_b, vprior, compat, x_bf16;
  double lam, a0, s0;
  const void* X;
  const int* y;
  int lik;              // AB_LIK_*
  float inv_var;        // AB_LIK_NORMAL: 1 / obs_var
  double ll_add;        // AB_LIK_NORMAL: N times the per-row normaliser, added once
  const float* yr;
};

struct HlrComp {
  int kind, P, idx_off, max_depth;
  double simlen, eps, mwg_var;
};

__device__ __forceinline__ float load_x(const HlrModelDev& m, size_t i) {
  if (m.x_bf16) return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(m.X)[i]);
  return __ldg(reinterpret_cast<const float*>(m.X) + i);
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
  const float yv = x - c;
  const float t = s + yv;
  c = (t - s) - yv;
  s = t;
}

// Stable log Bern(y | sigmoid(t)) and its derivative, FP32.
__device__ __forceinline__ void bern_terms(int y, float t, float& ll, float& r) {
  const float sp = fmaxf(t, 0.0f) + log1pf(__expf(-fabsf(t)));
  ll = y ? t - sp : -sp;
  const float sg = 1.0f / (1.0f + __expf(-t));
  r = (float)y - sg;
}

// Data factor of row n at t and its derivative in t, FP32: the logistic
// terms above, Poisson(exp(t)): y t - exp(t) - lgamma(y + 1) and y - exp(t)
// (the reference's y log(rate) - rate - sum_{k <= y} log k and its adjoint
// through exp), Normal(t, obs_var): -(y - t)^2 / (2 var) and (y - t) / var
// (the normaliser is added once per pass, ll_add).
__device__ __forceinline__ void lik_terms(const HlrModelDev& m, int n, float t, float& ll, float& r) {
  if (m.lik == AB_LIK_POISSON) {
    const int y = m.y[n];
    const float rate = expf(t);
    ll = (float)y * t - rate - lgammaf((float)y + 1.0f);
    r = (float)y - rate;
  } else if (m.lik == AB_LIK_NORMAL) {
    const float d = m.yr[n] - t;
    ll = -0.5f * d * d * m.inv_var;
    r = d * m.inv_var;
  } else {
    bern_terms(m.y[n], t, ll, r);
  }
}

// Shared-memory workspace of one chain CTA (sizes fixed by D).
struct Ws {
  double* par;     // [D+2]  current state
  double* prop;    // [D+2]  proposal state
  double* g;       // [D+1]  data gradient (theta..., b)
  double* blk_g;   // [D+2]  block gradient, block order
  double* p0;      // [D+2]  momentum at start
  double* ps;      // [D+2]  momentum working
  double* q;       // [D+2]  block position working
  double* aux1;    // [D+2]  spare (NUTS frontiers)
  double* aux2;    // [D+2]
  double* aux3;    // [D+2]
  double* aux4;    // [D+2]
  double* pt_ll;   // [D+2]  per-coordinate prior terms (log density)
  double* pt_dot;  // [D+2]  per-coordinate prior terms (d/dvar)
  double* gpart;   // [HLR_THREADS] per-thread partials (double)
  float* th;       // [D]    theta in FP32 for the data pass
  float* r;        // [HLR_CHUNK]
  double* red;     // [34]
  double* bcast;   // [8]   broadcast slots
  int* ibcast;     // [8]
};

__device__ __forceinline__ double cta_sum(double v, double* red) { return block_sum_f64(v, red); }

// Small-D pass widths: D gradient columns, the bias column, the
// log-likelihood; 16 columns for D + 2 <= 16, else 32.
constexpr int SMALL_COLS = 32;

// Sum over the warp's lanes of each of COLS per-lane values, transposed: on
// return v[0] of lane L holds the warp sum of column L % COLS (fixed
// butterfly order, so deterministic; COLS - 1 shuffles, plus one more round
// folding the two half-warps when COLS = 16).
template <int COLS>
__device__ __forceinline__ void warp_transpose_sum(double (&v)[COLS], int lane) {
#pragma unroll
  for (int sft = COLS / 2; sft >= 1; sft >>= 1) {
    const bool up = (lane & sft) != 0;
#pragma unroll
    for (int i = 0; i < sft; ++i) {
      const double send = up ? v[i] : v[i + sft];
      const double keep = up ? v[i + sft] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, sft);
    }
  }
  if (COLS == 16) v[0] += __shfl_xor_sync(0xffffffffu, v[0], 16);
}

// Data pass for D + 2 <= COLS: one row per thread (t, the log-likelihood term
// and the residual's contributions to all D + 1 gradient columns in
// registers, Kahan-compensated), then one transposed warp reduction and a
// fixed-order sum over the warps, all in FP64.  The row-per-thread walk
// keeps every thread busy at small N, where the segmented pass below is
// bound by its per-row shuffle latency.
template <int COLS>
__device__ double data_pass_small(const HlrModelDev& m, const double* par, Ws& ws, bool want_grad) {
  const int D = m.D, N = m.N;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int k = tid; k < D; k += blockDim.x) ws.th[k] = (float)par[k];
  const float bias = m.has_b ? (float)par[D] : 0.0f;
  __syncthreads();
  float th[COLS - 2];
#pragma unroll
  for (int k = 0; k < COLS - 2; ++k) th[k] = k < D ? ws.th[k] : 0.0f;
  float s[COLS], c[COLS];
#pragma unroll
  for (int j = 0; j < COLS; ++j) { s[j] = 0.0f; c[j] = 0.0f; }
  for (int n = tid; n < N; n += blockDim.x) {
    const size_t rb = (size_t)n * m.ldx;
    float x[COLS - 2];
    float t = 0.0f;
#pragma unroll
    for (int k = 0; k < COLS - 2; ++k) {
      x[k] = k < D ? load_x(m, rb + k) : 0.0f;
      t += x[k] * th[k];
    }
    float llv, rv;
    lik_terms(m, n, t + bias, llv, rv);
    kahan_add(s[COLS - 1], c[COLS - 1], llv);
    if (want_grad) {
#pragma unroll
      for (int k = 0; k < COLS - 2; ++k)
        if (k < D) kahan_add(s[k], c[k], rv * x[k]);
#pragma unroll
      for (int k = 0; k < COLS - 1; ++k)
        if (k == D) kahan_add(s[k], c[k], rv);
    }
  }
  double v[COLS];
#pragma unroll
  for (int j = 0; j < COLS; ++j) v[j] = (double)s[j] - (double)c[j];
  warp_transpose_sum<COLS>(v, lane);
  __syncthreads();
  if (lane < COLS) ws.gpart[warp * COLS + lane] = v[0];
  __syncthreads();
  if (tid < COLS) {
    double acc = 0.0;
    const int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; ++w) acc += ws.gpart[w * COLS + tid];
    if (tid == COLS - 1) ws.red[33] = acc;
    else if (want_grad && tid <= D) ws.g[tid] = acc;
  }
  __syncthreads();
  return ws.red[33];
}

// Data pass at `par` (theta in par[0..D-1], b = par[D] if has_b).  Writes
// ll_data (returned, all threads) and, if want_grad, ws.g[0..D] (theta then
// bias) — the full data gradient.
__device__ double data_pass(const HlrModelDev& m, const double* par, Ws& ws, bool want_grad) {
  const int D = m.D, N = m.N;
  if (D + 2 <= 16) return data_pass_small<16>(m, par, ws, want_grad);
  if (D + 2 <= SMALL_COLS) return data_pass_small<SMALL_COLS>(m, par, ws, want_grad);
  const int tid = threadIdx.x;
  for (int k = tid; k < D; k += blockDim.x) ws.th[k] = (float)par[k];
  const float bias = m.has_b ? (float)par[D] : 0.0f;
  __syncthreads();
  // segment of S lanes per row for the row dot products
  int S = 1;
  while (S < D && S < 32) S <<= 1;
  const int lane = tid & 31, warp = tid >> 5;
  const int segs_per_warp = 32 / S;
  const int seg = warp * segs_per_warp + lane / S;
  const int nseg = (blockDim.x >> 5) * segs_per_warp;
  const int ls = lane % S;
  // gradient accumulators: thread owns columns c = tid + i*blockDim (cols
  // D+1 including the bias column) for rows n = grp (mod ngrp)
  const int ncol = D + 1;
  const int ngrp = ncol >= (int)blockDim.x ? 1 : (int)blockDim.x / ncol;
  const int grp = ncol >= (int)blockDim.x ? 0 : tid / ncol;
  const int col0 = ncol >= (int)blockDim.x ? tid : tid % ncol;
  const bool gactive = grp < ngrp;
  float gs[HLR_MAX_COLS], gc[HLR_MAX_COLS];
#pragma unroll
  for (int i = 0; i < HLR_MAX_COLS; ++i) { gs[i] = 0.0f; gc[i] = 0.0f; }
  float lls = 0.0f, llc = 0.0f;
  for (int n0 = 0; n0 < N; n0 += HLR_CHUNK) {
    const int nc = min(HLR_CHUNK, N - n0);
    for (int i = seg; i < nc + ((nseg - nc % nseg) % nseg); i += nseg) {
      const int n = n0 + i;
      float part = 0.0f;
      if (i < nc) {
        const size_t rb = (size_t)n * m.ldx;
        for (int k = ls; k < D; k += S) part += load_x(m, rb + k) * ws.th[k];
      }
      for (int o = S >> 1; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if (ls == 0 && i < nc) {
        float llv, rv;
        lik_terms(m, n, part + bias, llv, rv);
        kahan_add(lls, llc, llv);
        ws.r[i] = rv;
      }
    }
    __syncthreads();
    if (want_grad && gactive) {
      for (int i = grp; i < nc; i += ngrp) {
        const float rv = ws.r[i];
        const size_t rb = (size_t)(n0 + i) * m.ldx;
#pragma unroll
        for (int j = 0; j < HLR_MAX_COLS; ++j) {
          const int c = col0 + j * (ncol >= (int)blockDim.x ? (int)blockDim.x : ncol);
          if (j > 0 && ncol < (int)blockDim.x) break;
          if (c < D) kahan_add(gs[j], gc[j], rv * load_x(m, rb + c));
          else if (c == D) kahan_add(gs[j], gc[j], rv);
        }
      }
    }
    __syncthreads();
  }
  const double ll = cta_sum((double)lls - (double)llc, ws.red);
  if (want_grad) {
    // combine the groups column by column in a fixed order
    const int stride = ncol >= (int)blockDim.x ? (int)blockDim.x : ncol;
    for (int j = 0; j < HLR_MAX_COLS; ++j) {
      const int c0 = j * stride;
      if (c0 >= ncol) break;
      ws.gpart[tid] = gactive ? (double)gs[j] - (double)gc[j] : 0.0;
      __syncthreads();
      if (ncol >= (int)blockDim.x) {
        const int c = c0 + tid;
        if (c < ncol) ws.g[c] = ws.gpart[tid];
      } else if (tid < ncol) {
        double acc = 0.0;
        for (int q = 0; q < ngrp; ++q) acc += ws.gpart[q * ncol + tid];
        ws.g[tid] = acc;
      }
      __syncthreads();
    }
  }
  return ll;
}

// ---- priors (binary64; reference formulas when compat) ----------------------
__device__ __forceinline__ double normal_ll(const HlrModelDev& m, double pt, double mean, double var) {
  const double t = pt - mean;
  if (m.compat) return var > 0.0 ? (-log(var)) - (0.5 * t * t / var) : -1e8;
  if (!(var > 0.0)) return -INFINITY;
  return -0.5 * log(2.0 * 3.14159265358979323846 * var) - 0.5 * t * t / var;
}
__device__ __forceinline__ double normal_dotarg2(const HlrModelDev& m, double pt, double mean, double var) {
  const double t = pt - mean;
  return m.compat ? (-0.5 * var) + (0.5 * (t * t) / (var * var))
                  : (-0.5 / var) + (0.5 * (t * t) / (var * var));
}
__device__ __forceinline__ double vprior_ll(const HlrModelDev& m, double v) {
  if (m.vprior == 0) return (m.lam > 0.0 && v > 0.0) ? log(m.lam) - m.lam * v : (m.compat ? -1e8 : -INFINITY);
  if (!(v > 0.0)) return m.compat ? -1e8 : -INFINITY;
  return m.a0 * log(m.s0) - lgamma(m.a0) - (m.a0 + 1.0) * log(v) - m.s0 / v;
}
__device__ __forceinline__ double vprior_dot(const HlrModelDev& m, double v) {
  if (m.vprior == 0) return (m.lam > 0.0 && v > 0.0) ? -m.lam : 0.0;
  return -(m.a0 + 1.0) / v + m.s0 / (v * v);
}

struct BlockInfo {
  bool th, b, v;
};

__device__ __forceinline__ BlockInfo block_info(const HlrModelDev& m, const int* idx, int P) {
  BlockInfo bi{false, false, false};
  for (int j = 0; j < P; ++j) {
    const int i = idx[j];
    if (i < m.D) bi.th = true;
    else if (i == m.D) bi.b = m.has_b != 0;
    else bi.v = true;
  }
  return bi;
}

// Full conditional of the block at `par` and (optionally) its gradient in
// block order into ws.blk_g.  Factor order as the generated ll_/grad_
// functions (CgLike.hs:139-147, CgGrad.hs:165-376).  All threads return ll.
__device__ double block_ll_grad(const HlrModelDev& m, const double* par, const int* idx, int P,
                                Ws& ws, bool want_grad) {
  const int D = m.D;
  const BlockInfo bi = block_info(m, idx, P);
  double data_ll = 0.0;
  if (bi.th || bi.b) data_ll = data_pass(m, par, ws, want_grad) + m.ll_add;
  const double b = m.has_b ? par[D] : 0.0, v = par[D + 1];
  // prior terms of the coefficients, one per thread; thread 0 then adds
  // them in the reference's (sequential) order
  if (bi.th || bi.v) {
    for (int k = threadIdx.x; k < D; k += blockDim.x) {
      ws.pt_ll[k] = normal_ll(m, par[k], 0.0, v);
      if (bi.v) ws.pt_dot[k] = normal_dotarg2(m, par[k], 0.0, v);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double ll = 0.0, gv = 0.0;
    if (bi.v) { ll += vprior_ll(m, v); gv += vprior_dot(m, v); }
    if (m.has_b && (bi.b || bi.v)) {
      ll += normal_ll(m, b, 0.0, v);
      if (bi.v) gv += normal_dotarg2(m, b, 0.0, v);
    }
    if (bi.th || bi.v) {
      double s = 0.0;
      for (int k = 0; k < D; ++k) {
        s += ws.pt_ll[k];
        if (bi.v) gv += ws.pt_dot[k];
      }
      ll += s;
    }
    ll += data_ll;
    ws.bcast[0] = ll;
    ws.bcast[1] = gv;
  }
  __syncthreads();
  const double ll = ws.bcast[0];
  if (want_grad) {
    const double gv = ws.bcast[1];
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
      const int i = idx[j];
      double gj;
      if (i < D) gj = -(par[i] - 0.0) / v + ws.g[i];                 // dotpt + data
      else if (i == D) gj = m.has_b ? -(b - 0.0) / v + ws.g[D] : 0.0;
      else gj = gv;
      ws.blk_g[j] = gj;
    }
  }
  __syncthreads();
  return ll;
}

__device__ __forceinline__ void set_block(double* par, const int* idx, int P, const double* q) {
  for (int j = threadIdx.x; j < P; j += blockDim.x) par[idx[j]] = q[j];
  __syncthreads();
}

// Sequential binary64 dot product in element order (thread 0), broadcast.
__device__ double seq_dot(const double* a, const double* b, int P, Ws& ws) {
  if (threadIdx.x == 0) {
    double acc = 0.0;
    for (int j = 0; j < P; ++j) acc += a[j] * b[j];
    ws.bcast[2] = acc;
  }
  __syncthreads();
  const double r = ws.bcast[2];
  __syncthreads();
  return r;
}

// ---- HMC: cbits/augur_mcmclib.h:343-424 -------------------------------------
__device__ int hmc_transition(const HlrModelDev& m, const HlrComp& cp, const int* idx, Ws& ws,
                              uint64_t seed, uint32_t iter, uint32_t chain, uint32_t ci,
                              double* cache_ll, bool* cache_ok) {
  const int P = cp.P;
  const int tid = threadIdx.x;
  for (int j = tid; j < P; j += blockDim.x) {
    Stream s = make_stream(seed, chain * (uint32_t)P + j, iter, TAG_MOM | (ci << 8));
    ws.p0[j] = s.normal();
  }
  if (tid == 0) {
    Stream h = make_stream(seed, chain, iter, TAG_HMC | (ci << 8));
    const double scale_eps = 0.8 + h.uniform() * (1.2 - 0.8);
    const double stepsize = scale_eps * cp.eps;
    const double sj = 0.9 + h.uniform() * (1.1 - 0.9);
    const unsigned rl = (unsigned)round(sj * cp.simlen / stepsize);
    ws.bcast[3] = stepsize;
    ws.ibcast[0] = (int)min(rl > 1u ? rl : 1u, 1u << 20);   // host bounds simlen/eps
    ws.bcast[4] = h.uniform();   // accept uniform (position 2)
  }
  for (int i = tid; i < m.D + 2; i += blockDim.x) ws.prop[i] = ws.par[i];
  __syncthreads();
  const double step = ws.bcast[3];
  const int L = ws.ibcast[0];
  const double u = ws.bcast[4];
  // gradient (and ll) at the current state
  const double ll_curr = block_ll_grad(m, ws.par, idx, P, ws, true);
  for (int j = tid; j < P; j += blockDim.x) {
    ws.ps[j] = __dadd_rn(ws.p0[j], __dmul_rn(step / 2.0, ws.blk_g[j]));
    ws.q[j] = ws.par[idx[j]];
  }
  __syncthreads();
  double ll_prop = 0.0;
  for (int l = 0; l < L; ++l) {
    for (int j = tid; j < P; j += blockDim.x) ws.q[j] = __dadd_rn(ws.q[j], __dmul_rn(step, ws.ps[j]));
    __syncthreads();
    set_block(ws.prop, idx, P, ws.q);
    if (l != L - 1) {
      block_ll_grad(m, ws.prop, idx, P, ws, true);
      for (int j = tid; j < P; j += blockDim.x) ws.ps[j] = __dadd_rn(ws.ps[j], __dmul_rn(step, ws.blk_g[j]));
      __syncthreads();
    }
  }
  ll_prop = block_ll_grad(m, ws.prop, idx, P, ws, true);
  for (int j = tid; j < P; j += blockDim.x) ws.ps[j] = __dadd_rn(ws.ps[j], __dmul_rn(step / 2.0, ws.blk_g[j]));
  __syncthreads();
  const double k0 = seq_dot(ws.p0, ws.p0, P, ws);
  const double k1 = seq_dot(ws.ps, ws.ps, P, ws);
  const double auxll = k0 / 2.0 - k1 / 2.0;
  const double dlog = ll_prop - ll_curr + auxll;   // minus the energy error
  const int acc = log(u) < dlog;
  // divergent: the energy error passed the bound, or is not finite
  const int div = !(dlog > -AB_DIVERGENCE_DH);
  if (acc)
    for (int i = tid; i < m.D + 2; i += blockDim.x) ws.par[i] = ws.prop[i];
  __syncthreads();
  (void)cache_ll; (void)cache_ok;
  return acc | (div << 1);
}

// ---- NUTS: cbits/augur_mcmclib.h:575-776 (iterative restatement) ------------
// Stacks live in global scratch: [3][HLR_STK][P] doubles per chain.
struct NutsFrame {
  int j, phase, ln, ls;
};

__device__ int nuts_update_s(int s, const double* tp, const double* mp, const double* tm,
                             const double* mm, int P, Ws& ws) {
  int res = 0;
  if (s == 1) {
    for (int j = threadIdx.x; j < P; j += blockDim.x) ws.blk_g[j] = __dadd_rn(tp[j], __dmul_rn(-1.0, tm[j]));
    __syncthreads();
    const double d1 = seq_dot(ws.blk_g, mp, P, ws);
    const double d2 = seq_dot(ws.blk_g, mm, P, ws);
    res = (d1 >= 0.0 && d2 >= 0.0) ? 1 : 0;
  }
  return res;
}

__device__ int nuts_transition(const HlrModelDev& m, const HlrComp& cp, const int* idx, Ws& ws,
                               double* stk, uint64_t seed, uint32_t iter, uint32_t chain, uint32_t ci,
                               int* depth_out, int* leaves_out, int* error_out, int* div_out) {
  const int P = cp.P;
  const int tid = threadIdx.x;
  double* tp_stk = stk;                          // theta_prop stack
  double* ts_stk = stk + (size_t)HLR_STK * P;    // theta stack
  double* ms_stk = stk + (size_t)2 * HLR_STK * P;  // mom stack
  double* th0 = ws.aux1;   // theta0 (block)
  double* thm = ws.aux2;   // theta_minus
  double* thp = ws.aux3;   // theta_plus
  double* thprop = ws.q;   // working theta
  double* mm = ws.p0;      // mom_minus
  double* mp = ws.ps;      // mom_plus
  double* aux4 = ws.aux4;  // spare copy buffer
  // initialise
  for (int j = tid; j < P; j += blockDim.x) {
    th0[j] = ws.par[idx[j]];
    thm[j] = th0[j];
    thp[j] = th0[j];
    Stream s = make_stream(seed, chain * (uint32_t)P + j, iter, TAG_MOM | (ci << 8));
    mm[j] = s.normal();
    mp[j] = mm[j];
  }
  for (int i = tid; i < m.D + 2; i += blockDim.x) ws.prop[i] = ws.par[i];
  __syncthreads();
  // h substream position counter lives in ibcast[1] (read/advanced by thread 0)
  const double ll0 = block_ll_grad(m, ws.par, idx, P, ws, false);
  const double mm2 = seq_dot(mm, mm, P, ws);
  if (tid == 0) {
    Stream h = make_stream(seed, chain, iter, TAG_NUTS | (ci << 8));
    const double e = -1.0 * log(h.uniform());
    ws.bcast[5] = ll0 - 0.5 * mm2 - e;   // logu
    ws.ibcast[1] = (int)h.pos;
    ws.ibcast[2] = -1; ws.ibcast[3] = -1; ws.ibcast[4] = -1;  // tp, ts, ms stack heads
    ws.ibcast[5] = 0;  // leaves
    ws.ibcast[6] = 0;  // overflow flag
    ws.ibcast[7] = 0;  // divergence flag
  }
  __syncthreads();
  const double logu = ws.bcast[5];
  auto draw_u = [&]() -> double {   // next uniform of the sequential h stream (uniform across threads)
    __syncthreads();
    if (tid == 0) {
      Stream h = make_stream(seed, chain, iter, TAG_NUTS | (ci << 8));
      h.pos = (uint32_t)ws.ibcast[1];
      ws.bcast[6] = h.uniform();
      ws.ibcast[1] = (int)h.pos;
    }
    __syncthreads();
    const double r = ws.bcast[6];
    __syncthreads();
    return r;
  };
  auto push = [&](double* base, int head_slot, const double* v) {
    __syncthreads();
    int hd = ws.ibcast[head_slot] + 1;
    if (hd >= HLR_STK) { if (tid == 0) ws.ibcast[6] = 1; hd = HLR_STK - 1; }
    for (int j = tid; j < P; j += blockDim.x) base[(size_t)hd * P + j] = v[j];
    __syncthreads();
    if (tid == 0) ws.ibcast[head_slot] = hd;
    __syncthreads();
  };
  auto head = [&](int head_slot) -> int {
    const int h = ws.ibcast[head_slot];
    return h < 0 ? 0 : h;
  };
  auto pop = [&](int head_slot) -> int {   // returns the popped slot index
    __syncthreads();
    const int h = ws.ibcast[head_slot];
    __syncthreads();
    if (tid == 0) ws.ibcast[head_slot] = h - 1;
    __syncthreads();
    return h < 0 ? 0 : h;
  };
  int n = 1, jd = 0, s = 1;
  double stepsize = cp.eps;
  NutsFrame fr[24];
  for (;;) {
    int f_cpy = 0;
    if (tid == 0) { ws.ibcast[3] = -1; ws.ibcast[4] = -1; }
    __syncthreads();
    const int dir = draw_u() < 0.5 ? 0 : 1;   // 0 = MINUS
    stepsize = dir == 0 ? -cp.eps : cp.eps;
    double* mom = dir == 0 ? mm : mp;
    for (int j = tid; j < P; j += blockDim.x) thprop[j] = dir == 0 ? thm[j] : thp[j];
    __syncthreads();
    // ---- build_tree(thprop, mom, jd, dir) as an explicit post-order walk
    int sp = 0;
    fr[0].j = jd; fr[0].phase = 0;
    int rn = 0, rs = 0;       // return value of the last finished subtree
    while (sp >= 0) {
      NutsFrame& F = fr[sp];
      if (F.j == 0) {
        // leaf: leapfrog1 (:305-325) - gradient, half kick, drift, gradient, half kick
        set_block(ws.prop, idx, P, thprop);
        block_ll_grad(m, ws.prop, idx, P, ws, true);
        for (int j = tid; j < P; j += blockDim.x) {
          mom[j] = __dadd_rn(mom[j], __dmul_rn(stepsize / 2.0, ws.blk_g[j]));
          thprop[j] = __dadd_rn(thprop[j], __dmul_rn(stepsize, mom[j]));
        }
        __syncthreads();
        set_block(ws.prop, idx, P, thprop);
        const double llp = block_ll_grad(m, ws.prop, idx, P, ws, true);
        for (int j = tid; j < P; j += blockDim.x) mom[j] = __dadd_rn(mom[j], __dmul_rn(stepsize / 2.0, ws.blk_g[j]));
        __syncthreads();
        if (tid == 0) ws.ibcast[5] += 1;
        push(tp_stk, 2, thprop);
        const double ll = llp - 0.5 * seq_dot(mom, mom, P, ws);
        rn = logu <= ll ? 1 : 0;
        rs = logu < 1000.0 + ll ? 1 : 0;
        // a leaf outside the slice by the reference's deltaMax (1000) ends
        // the tree: the iteration counts as divergent
        if (tid == 0 && !rs) ws.ibcast[7] = 1;
        --sp;
        continue;
      }
      if (F.phase == 0) {
        F.phase = 1;
        fr[sp + 1].j = F.j - 1; fr[sp + 1].phase = 0;
        ++sp;
        continue;
      }
      if (F.phase == 1) {             // left subtree finished
        F.ln = rn; F.ls = rs;
        if (F.ls == 1) {
          if (F.j == 1) { push(ts_stk, 3, thprop); push(ms_stk, 4, mom); }
          F.phase = 2;
          fr[sp + 1].j = F.j - 1; fr[sp + 1].phase = 0;
          ++sp;
        } else {
          rn = F.ln; rs = F.ls;
          --sp;
        }
        continue;
      }
      // phase 2: right subtree finished (rn, rs)
      const int p1 = pop(2);
      const int p2 = pop(2);
      const double bias = ((double)rn) / (F.ln + rn);
      const double uu = draw_u();
      // push(prop2) or push(prop1): copy through the spare buffer
      const int src = (uu < bias) ? p1 : p2;
      for (int j = tid; j < P; j += blockDim.x) aux4[j] = tp_stk[(size_t)src * P + j];
      push(tp_stk, 2, aux4);
      F.ln += rn;
      const double* tpv; const double* mpv; const double* tmv; const double* mmv;
      const int th_slot = head(3), mo_slot = head(4);
      if (dir == 0) { tpv = ts_stk + (size_t)th_slot * P; mpv = ms_stk + (size_t)mo_slot * P; tmv = thprop; mmv = mom; }
      else { tmv = ts_stk + (size_t)th_slot * P; mmv = ms_stk + (size_t)mo_slot * P; tpv = thprop; mpv = mom; }
      F.ls = nuts_update_s(rs, tpv, mpv, tmv, mmv, P, ws);
      if (F.j > 1) { pop(3); pop(4); }
      rn = F.ln; rs = F.ls;
      --sp;
    }
    // ---- outer loop body (:744-774)
    if (dir == 0) for (int j = tid; j < P; j += blockDim.x) thm[j] = thprop[j];
    else for (int j = tid; j < P; j += blockDim.x) thp[j] = thprop[j];
    __syncthreads();
    const int pp = pop(2);
    if (rs == 1) {
      const unsigned ratio = (unsigned)(((double)rn) / n);   // augur_min is unsigned
      const double bias = (double)(ratio < 1u ? ratio : 1u);
      if (draw_u() < bias) {
        for (int j = tid; j < P; j += blockDim.x) thprop[j] = tp_stk[(size_t)pp * P + j];
        f_cpy = 1;
      }
      __syncthreads();
    }
    n += rn;
    s = nuts_update_s(rs, thp, mp, thm, mm, P, ws);
    jd += 1;
    if (s != 1 || jd >= cp.max_depth || ws.ibcast[6]) {
      if (f_cpy) for (int j = tid; j < P; j += blockDim.x) th0[j] = thprop[j];
      __syncthreads();
      break;
    }
  }
  set_block(ws.par, idx, P, th0);
  if (tid == 0) {
    *depth_out = jd;
    *leaves_out = ws.ibcast[5];
    *error_out = ws.ibcast[6];
    *div_out = ws.ibcast[7];
  }
  __syncthreads();
  return 0;
}

// ---- Reflective slice: cbits/augur_mcmclib.h:498-543 ------------------------
// Momentum from (c*P + j, iter, MOM|ci<<8); slice level z = ll(curr) - Exp(1)
// with the exponential from (c, iter, RSLICE|ci<<8); augur_max(1,
// round(simlen / eps)) steps of q += eps p0, each followed by the log density
// at the new point and, outside the slice, a reflection of p0 off the block
// gradient there (p0 += -2 (p0.g)/(g.g) g, sequential dot products).  The
// move is kept only if the last point is inside the slice.
__device__ int rslice_transition(const HlrModelDev& m, const HlrComp& cp, const int* idx, Ws& ws,
                                 uint64_t seed, uint32_t iter, uint32_t chain, uint32_t ci, int* refl_out) {
  const int P = cp.P;
  const int tid = threadIdx.x;
  for (int j = tid; j < P; j += blockDim.x) {
    Stream s = make_stream(seed, chain * (uint32_t)P + j, iter, TAG_MOM | (ci << 8));
    ws.p0[j] = s.normal();
  }
  if (tid == 0) {
    Stream h = make_stream(seed, chain, iter, TAG_RSLICE | (ci << 8));
    ws.bcast[3] = -1.0 * log(h.uniform());
    const unsigned rl = (unsigned)round(cp.simlen / cp.eps);
    ws.ibcast[0] = (int)min(rl > 1u ? rl : 1u, 1u << 20);   // host bounds simlen/eps
  }
  for (int i = tid; i < m.D + 2; i += blockDim.x) ws.prop[i] = ws.par[i];
  __syncthreads();
  const double expo = ws.bcast[3];
  const int L = ws.ibcast[0];
  const double step = cp.eps;
  const double z = block_ll_grad(m, ws.par, idx, P, ws, false) - expo;
  for (int j = tid; j < P; j += blockDim.x) ws.q[j] = ws.par[idx[j]];
  __syncthreads();
  bool cond = false;
  int refl = 0;
  for (int l = 0; l < L; ++l) {
    for (int j = tid; j < P; j += blockDim.x) ws.q[j] = __dadd_rn(ws.q[j], __dmul_rn(step, ws.p0[j]));
    __syncthreads();
    set_block(ws.prop, idx, P, ws.q);
    cond = block_ll_grad(m, ws.prop, idx, P, ws, false) < z;    // same value on every thread
    if (cond) {
      block_ll_grad(m, ws.prop, idx, P, ws, true);
      const double a1 = seq_dot(ws.p0, ws.blk_g, P, ws);
      const double a2 = seq_dot(ws.blk_g, ws.blk_g, P, ws);
      const double sc = __dmul_rn(-2.0, a1 / a2);
      for (int j = tid; j < P; j += blockDim.x) ws.p0[j] = __dadd_rn(ws.p0[j], __dmul_rn(sc, ws.blk_g[j]));
      __syncthreads();
      ++refl;
    }
  }
  if (!cond)
    for (int i = tid; i < m.D + 2; i += blockDim.x) ws.par[i] = ws.prop[i];
  __syncthreads();
  *refl_out = refl;
  return !cond;
}

// ---- MWG on one scalar of par: augur_mcmclib.h:89-105,178-193 ---------------
__device__ int mwg_transition(const HlrModelDev& m, const HlrComp& cp, const int* idx, Ws& ws,
                              uint64_t seed, uint32_t iter, uint32_t chain, uint32_t ci) {
  const int which = idx[0];
  if (threadIdx.x == 0) {
    Stream s = make_stream(seed, chain, iter, TAG_MWG | (ci << 8));
    const double x = ws.par[which];
    const double xp = x + sqrt(cp.mwg_var) * s.normal();
    ws.bcast[3] = xp;
    ws.bcast[4] = s.uniform();
    ws.bcast[5] = m.compat ? normal_ll(m, x, x, cp.mwg_var) - normal_ll(m, xp, x, cp.mwg_var) : 0.0;
  }
  for (int i = threadIdx.x; i < m.D + 2; i += blockDim.x) ws.prop[i] = ws.par[i];
  __syncthreads();
  if (threadIdx.x == 0) ws.prop[which] = ws.bcast[3];
  __syncthreads();
  const double lc = block_ll_grad(m, ws.par, idx, 1, ws, false);
  const double lp = block_ll_grad(m, ws.prop, idx, 1, ws, false);
  const int acc = log(ws.bcast[4]) < lp - lc + ws.bcast[5];
  if (acc && threadIdx.x == 0) ws.par[which] = ws.prop[which];
  __syncthreads();
  return acc;
}

__device__ Ws carve(void* base, int D) {
  Ws w;
  double* d = reinterpret_cast<double*>(base);
  const int V = D + 2;
  w.par = d; d += V; w.prop = d; d += V; w.g = d; d += V; w.blk_g = d; d += V;
  w.p0 = d; d += V; w.ps = d; d += V; w.q = d; d += V; w.aux1 = d; d += V; w.aux2 = d; d += V;
  w.aux3 = d; d += V; w.aux4 = d; d += V;
  w.pt_ll = d; d += V; w.pt_dot = d; d += V;
  w.gpart = d; d += HLR_THREADS;
  w.red = d; d += 34;
  w.bcast = d; d += 8;
  w.ibcast = reinterpret_cast<int*>(d); d += 8;
  w.th = reinterpret_cast<float*>(d); d += (D + 1) / 2 + 1;
  w.r = reinterpret_cast<float*>(d);
  return w;
}

size_t hlr_smem_bytes(int D) {
  const int V = D + 2;
  return sizeof(double) * (13 * (size_t)V + HLR_THREADS + 34 + 8 + 8 + (D + 1) / 2 + 1) +
         sizeof(float) * HLR_CHUNK;
}

// One CTA per chain: n_iter iterations of the schedule `comps`.
// stats[c][ci][5] = {accepts, sum depth, sum leaves, errors, divergent iterations}.
__global__ void __launch_bounds__(HLR_THREADS)
hlr_chain_kernel(HlrModelDev m, const HlrComp* __restrict__ comps, int n_comps,
                 const int* __restrict__ idx_all, double* __restrict__ pars, int n_iter,
                 uint32_t iter0, uint64_t seed, double* __restrict__ stats,
                 double* __restrict__ nuts_stk, int stk_P) {
  extern __shared__ double smem_d[];
  Ws ws = carve(smem_d, m.D);
  const int c = blockIdx.x;
  double* par_g = pars + (size_t)c * (m.D + 2);
  for (int i = threadIdx.x; i < m.D + 2; i += blockDim.x) ws.par[i] = par_g[i];
  __syncthreads();
  for (int it = 0; it < n_iter; ++it) {
    const uint32_t iter = iter0 + (uint32_t)it;
    for (int ci = 0; ci < n_comps; ++ci) {
      const HlrComp cp = comps[ci];
      const int* idx = idx_all + cp.idx_off;
      double* st = stats + ((size_t)c * n_comps + ci) * AB_HLR_STATS;
      if (cp.kind == COMP_HMC) {
        const int a = hmc_transition(m, cp, idx, ws, seed, iter, (uint32_t)c, (uint32_t)ci, nullptr, nullptr);
        if (threadIdx.x == 0) { st[0] += a & 1; st[4] += a >> 1; }
      } else if (cp.kind == COMP_NUTS) {
        __shared__ int sh_out[4];
        nuts_transition(m, cp, idx, ws, nuts_stk + (size_t)c * 3 * HLR_STK * stk_P, seed, iter,
                        (uint32_t)c, (uint32_t)ci, &sh_out[0], &sh_out[1], &sh_out[2], &sh_out[3]);
        if (threadIdx.x == 0) { st[1] += sh_out[0]; st[2] += sh_out[1]; st[3] += sh_out[2]; st[4] += sh_out[3]; }
      } else if (cp.kind == COMP_RSLICE) {
        int refl = 0;
        const int a = rslice_transition(m, cp, idx, ws, seed, iter, (uint32_t)c, (uint32_t)ci, &refl);
        if (threadIdx.x == 0) { st[0] += a; st[2] += refl; }
      } else {
        const int a = mwg_transition(m, cp, idx, ws, seed, iter, (uint32_t)c, (uint32_t)ci);
        if (threadIdx.x == 0) st[0] += a;
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < m.D + 2; i += blockDim.x) par_g[i] = ws.par[i];
}

// Log-density and gradient of a block for C parameter vectors (one CTA per
// vector): the data pass and priors used by the transitions, exposed for
// parity checks and for callers that drive their own samplers.
__global__ void __launch_bounds__(HLR_THREADS)
hlr_ll_grad_kernel(HlrModelDev m, const int* __restrict__ idx, int P, const double* __restrict__ pars,
                   double* __restrict__ ll, double* __restrict__ grad) {
  extern __shared__ double smem_d[];
  Ws ws = carve(smem_d, m.D);
  const int c = blockIdx.x;
  for (int i = threadIdx.x; i < m.D + 2; i += blockDim.x) ws.par[i] = pars[(size_t)c * (m.D + 2) + i];
  __syncthreads();
  const double l = block_ll_grad(m, ws.par, idx, P, ws, grad != nullptr);
  if (threadIdx.x == 0) ll[c] = l;
  if (grad != nullptr)
    for (int j = threadIdx.x; j < P; j += blockDim.x) grad[(size_t)c * P + j] = ws.blk_g[j];
}

static int make_model(HlrModelDev& m, const ab_hlr_model* d) {
  AB_REQUIRE(d != nullptr, AB_ERR_ARG, "hlr: null model");
  AB_REQUIRE(d->N > 0 && d->D > 0 && d->D <= HLR_MAX_D, AB_ERR_ARG,
             "hlr: need N > 0 and 0 < D <= %d (N=%d D=%d)", HLR_MAX_D, d->N, d->D);
  AB_REQUIRE(d->lik == AB_LIK_BERNOULLI || d->lik == AB_LIK_POISSON || d->lik == AB_LIK_NORMAL, AB_ERR_ARG,
             "hlr: unknown likelihood %d", d->lik);
  AB_REQUIRE(d->X && (d->lik == AB_LIK_NORMAL ? d->yr != nullptr : d->y != nullptr), AB_ERR_ARG,
             "hlr: null data pointer");
  AB_REQUIRE(d->lik != AB_LIK_NORMAL || d->obs_var > 0.0, AB_ERR_ARG, "hlr: the observation variance must be > 0");
  AB_REQUIRE(d->x_dtype == AB_F32 || d->x_dtype == AB_BF16, AB_ERR_ARG, "hlr: X must be f32 or bf16");
  AB_REQUIRE(d->ldx >= d->D, AB_ERR_ARG, "hlr: ldx < D");
  AB_REQUIRE(d->vprior == 0 || d->vprior == 1, AB_ERR_ARG, "hlr: vprior must be 0 or 1");
  m.N = d->N; m.D = d->D; m.ldx = d->ldx; m.has_b = d->has_b != 0; m.vprior = d->vprior;
  m.compat = d->compat != 0; m.x_bf16 = d->x_dtype == AB_BF16;
  m.lam = d->lam; m.a0 = d->a0; m.s0 = d->s0; m.X = d->X; m.y = d->y;
  m.lik = d->lik;
  m.yr = d->yr;
  m.inv_var = d->lik == AB_LIK_NORMAL ? (float)(1.0 / d->obs_var) : 0.0f;
  // per-row Normal normaliser: the reference's -log(var) (compat) or -log(2 pi var) / 2
  m.ll_add = d->lik != AB_LIK_NORMAL ? 0.0
             : (double)d->N * (m.compat ? -log(d->obs_var) : -0.5 * log(2.0 * M_PI * d->obs_var));
  return AB_OK;
}

static int check_idx_host(const int* idx_host, int P, int D) {
  for (int j = 0; j < P; ++j)
    AB_REQUIRE(idx_host[j] >= 0 && idx_host[j] < D + 2, AB_ERR_ARG, "hlr: block index %d out of range", idx_host[j]);
  return AB_OK;
}

}  // namespace ab

using namespace ab;

extern "C" size_t ab_hlr_chain_scratch_bytes(int C, int D) {
  return sizeof(double) * (size_t)C * 3 * HLR_STK * (size_t)(D + 2);
}

extern "C" int ab_hlr_ll_grad(const ab_hlr_model* model, const int* idx_dev, const int* idx_host, int P,
                              int C, const double* pars, double* ll, double* grad, void* stream) {
  HlrModelDev m;
  int rc = make_model(m, model);
  if (rc) return rc;
  AB_REQUIRE(C > 0 && P > 0 && P <= m.D + 2, AB_ERR_ARG, "ab_hlr_ll_grad: bad C or P");
  AB_REQUIRE(idx_dev && idx_host && pars && ll, AB_ERR_ARG, "ab_hlr_ll_grad: null pointer");
  rc = check_idx_host(idx_host, P, m.D);
  if (rc) return rc;
  const size_t smem = hlr_smem_bytes(m.D);
  AB_CUDA(cudaFuncSetAttribute(hlr_ll_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  hlr_ll_grad_kernel<<<C, HLR_THREADS, smem, as_stream(stream)>>>(m, idx_dev, P, pars, ll, grad);
  AB_LAUNCH_CHECK("hlr_ll_grad_kernel");
  return AB_OK;
}

extern "C" int ab_hlr_run_chains(const ab_hlr_model* model, const ab_hlr_comp* comps_host,
                                 const void* comps_dev, int n_comps, const int* idx_dev,
                                 const int* idx_host, int C, double* pars, int n_iter, uint32_t iter0,
                                 uint64_t seed, double* stats, void* scratch, void* stream) {
  HlrModelDev m;
  int rc = make_model(m, model);
  if (rc) return rc;
  AB_REQUIRE(C > 0 && n_iter >= 0, AB_ERR_ARG, "ab_hlr_run_chains: bad C or n_iter");
  AB_REQUIRE(n_comps > 0 && n_comps <= HLR_MAX_COMPS, AB_ERR_ARG, "ab_hlr_run_chains: 1..%d components",
             HLR_MAX_COMPS);
  AB_REQUIRE(comps_host && comps_dev && idx_dev && idx_host && pars && stats, AB_ERR_ARG,
             "ab_hlr_run_chains: null pointer");
  bool has_nuts = false;
  for (int i = 0; i < n_comps; ++i) {
    const ab_hlr_comp& c = comps_host[i];
    AB_REQUIRE(c.kind >= 0 && c.kind <= 3, AB_ERR_ARG, "component %d: unknown kind", i);
    AB_REQUIRE(c.P > 0 && c.P <= m.D + 2, AB_ERR_ARG, "component %d: bad block size", i);
    AB_REQUIRE(c.kind != 2 || c.P == 1, AB_ERR_ARG, "component %d: MWG moves one scalar", i);
    AB_REQUIRE(c.kind == 2 || c.eps > 0.0, AB_ERR_ARG, "component %d: step size must be > 0", i);
    AB_REQUIRE((c.kind != 0 && c.kind != 3) || (c.simlen >= 0.0 && c.simlen / c.eps <= 1e5), AB_ERR_ARG,
               "component %d: HMC / RSlice simlen/eps must be <= 1e5 steps", i);
    AB_REQUIRE(c.kind != 2 || c.mwg_var > 0.0, AB_ERR_ARG, "component %d: MWG variance must be > 0", i);
    AB_REQUIRE(c.kind != 1 || (c.max_depth > 0 && c.max_depth <= 14), AB_ERR_ARG,
               "component %d: NUTS max_depth must be 1..14", i);
    rc = check_idx_host(idx_host + c.idx_off, c.P, m.D);
    if (rc) return rc;
    has_nuts |= c.kind == 1;
  }
  AB_REQUIRE(!has_nuts || scratch, AB_ERR_ARG, "ab_hlr_run_chains: NUTS needs scratch");
  static_assert(sizeof(ab_hlr_comp) == sizeof(HlrComp), "component layout");
  const size_t smem = hlr_smem_bytes(m.D);
  AB_REQUIRE(smem <= 200 * 1024, AB_ERR_ARG, "hlr: D too large for the per-chain engine");
  AB_CUDA(cudaFuncSetAttribute(hlr_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  hlr_chain_kernel<<<C, HLR_THREADS, smem, as_stream(stream)>>>(
      m, reinterpret_cast<const HlrComp*>(comps_dev), n_comps, idx_dev, pars, n_iter, iter0, seed, stats,
      reinterpret_cast<double*>(scratch), m.D + 2);
  AB_LAUNCH_CHECK("hlr_chain_kernel");
  return AB_OK;
}
