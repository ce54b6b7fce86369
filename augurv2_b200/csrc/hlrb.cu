// Batched HLR log density and gradient on the tensor cores: C chains against
// one data set, each chain's FP32 parameter vector theta[c][0..D-1].
//
//   logp(theta) = sum_n [ y_n t_n - softplus(t_n) ] + sum_d log prior(theta_d),
//   t = X theta,   grad = X^T (y - sigmoid(t)) + d/dtheta log prior
//
// which is the reference's generated ll/grad pair for the HLR model
// (compiler/augur/src/Comm/CgLike.hs:139-147 over augur_bernoulli_ll,
// augur_dist.c:59-66, and CgGrad.hs:345-376 with augur_bernoulli_dotarg1 x
// augur_expit_grad_0, augur_dist.c:68-71, augur_math.c:56-59) evaluated for
// all chains at once:
//
//   forward  T^T[C x N] = Theta3[C x 3D] . X[N x D]^T   (theta split hi+mid+lo
//            into bf16, so the FP32 product is exact to FP32 rounding); the
//            epilogue turns each t into its log-likelihood term (summed per
//            chain, 128-row tile and column group, Kahan-compensated) and the
//            residual r = y - sigmoid(t), stored as two bf16 parts (hi + mid,
//            within 2^-18 of r: the gradient's per-term error bound stays
//            below its 1e-5 tolerance against |g| + sum_n |r_n x_n|, and the
//            gradient only steers leapfrog steps, whose accept test uses the
//            FP32-exact log density);
//   backward G[C x D] = sum_p R_p[C x N] . Xt[D x N]^T, split over rows into
//            deterministic FP32 partial tiles;
//   finish   one block per chain: FP64 sums of the per-tile log-likelihood
//            partials and of the gradient partials in a fixed order, plus
//            the FP64 prior and its gradient.
// X is bf16 [N][ldx].  The backward operands are stored K-blocked so that
// every 128 x 64 tile the tensor memory accelerator fetches is one
// contiguous 16 KB box (row-major [rows][N] tiles would touch 128 rows that
// lie megabytes apart):
//   Xt  [Np/64][D][64]     the transpose of X in 64-row blocks, zero padded
//                          (Np = N rounded up to 64), built once by
//                          ab_hlrb_transpose;
//   R2  [Np/64][2][C][64]  the residual parts, written by the forward pass.
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"
#include "tc_gemm.cuh"
#include "tc_group.cuh"
#include "tc_host.cuh"

namespace ab {
namespace {

constexpr int FWD_BN_DEFAULT = 256;   // data rows per forward tile (launch shape: 128 or 256)
constexpr int R_PARTS = 2;          // bf16 parts of the residual
constexpr int FWD_MAX_GROUPS = 4;   // column groups of the forward epilogue (16 warps)
// gradient columns per backward tile by default: the narrowest of 32 / 64 /
// 128 that covers D (wider D takes several 128-column tiles)
inline int bwd_bn(int D) { return D <= 32 ? 32 : (D <= 64 ? 64 : 128); }

inline int round_up(int a, int b) { return (a + b - 1) / b * b; }
inline size_t align256(size_t a) { return (a + 255) & ~size_t(255); }

// Launch shape of one pass: the built-in choice, or the fields a caller (the
// autotuner) set in ab_hlrb_config.
struct Launch {
  int fwd_warps, bn, splits, fwd_bn;
};

struct Layout {
  int Np, Dp, fwd_tiles, groups, splits, ldw, bn, fwd_bn;
  size_t off_t3, off_r3, off_ll, off_w, total;
};

int check_config(const ab_hlrb_config* cfg) {
  if (!cfg) return AB_OK;
  AB_REQUIRE(cfg->fwd_warps == 0 || cfg->fwd_warps == 4 || cfg->fwd_warps == 8 || cfg->fwd_warps == 16,
             AB_ERR_ARG, "hlrb: fwd_warps must be 0, 4, 8 or 16 (got %d)", cfg->fwd_warps);
  AB_REQUIRE(cfg->bwd_bn == 0 || cfg->bwd_bn == 32 || cfg->bwd_bn == 64 || cfg->bwd_bn == 128, AB_ERR_ARG,
             "hlrb: bwd_bn must be 0, 32, 64 or 128 (got %d)", cfg->bwd_bn);
  AB_REQUIRE(cfg->bwd_splits >= 0, AB_ERR_ARG, "hlrb: bwd_splits must be >= 0 (got %d)", cfg->bwd_splits);
  AB_REQUIRE(cfg->fwd_bn == 0 || cfg->fwd_bn == 128 || cfg->fwd_bn == 256, AB_ERR_ARG,
             "hlrb: fwd_bn must be 0, 128 or 256 (got %d)", cfg->fwd_bn);
  return AB_OK;
}

Layout layout(int N, int D, int C, const ab_hlrb_config* cfg) {
  Launch q{8, bwd_bn(D), 0, FWD_BN_DEFAULT};
  if (cfg) {
    if (cfg->fwd_warps) q.fwd_warps = cfg->fwd_warps;
    if (cfg->fwd_bn) q.fwd_bn = cfg->fwd_bn;
    if (cfg->bwd_bn) q.bn = cfg->bwd_bn;
    q.splits = cfg->bwd_splits;
  }
  Layout L;
  L.Np = round_up(N, 64);
  L.Dp = round_up(D, 64);
  L.fwd_bn = q.fwd_bn;
  L.fwd_tiles = (N + L.fwd_bn - 1) / L.fwd_bn;
  L.groups = q.fwd_warps / 4;
  L.bn = q.bn;
  const int tiles = ((C + tc::BM - 1) / tc::BM) * ((D + L.bn - 1) / L.bn);
  const int kb = L.Np / tc::BK;
  int sp = q.splits > 0 ? q.splits : tc::sm_count() / tiles;
  if (sp < 1) sp = 1;
  if (sp > kb) sp = kb;
  // the kernel's own split arithmetic (whole K steps per split)
  const int per = (kb + sp - 1) / sp;
  L.splits = (kb + per - 1) / per;
  L.ldw = round_up(D, 32);
  size_t o = 0;
  L.off_t3 = o;
  o = align256(o + (size_t)C * 3 * L.Dp * 2);
  L.off_r3 = o;
  o = align256(o + (size_t)C * R_PARTS * L.Np * 2);
  L.off_ll = o;
  o = align256(o + (size_t)L.fwd_tiles * FWD_MAX_GROUPS * C * 4);
  L.off_w = o;
  o = align256(o + (size_t)L.splits * C * L.ldw * 4);
  L.total = o;
  return L;
}

__device__ __forceinline__ void split3(float x, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
  h = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h);   // exact in FP32
  m = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(m);  // exact in FP32
  l = __float2bfloat16_rn(r2);
}

// theta [C][ldt] f32 -> Theta3 [C][3][Dp] bf16 (hi, mid, lo; zero padding).
__device__ __forceinline__ void split_elem(int c, int d, int D, int Dp, const float* __restrict__ theta, int ldt,
                                          __nv_bfloat16* __restrict__ t3) {
  __nv_bfloat16 h, m, l;
  if (d < D) {
    split3(theta[(size_t)c * ldt + d], h, m, l);
  } else {
    h = m = l = __float2bfloat16_rn(0.0f);
  }
  __nv_bfloat16* row = t3 + (size_t)c * 3 * Dp;
  row[d] = h;
  row[Dp + d] = m;
  row[2 * Dp + d] = l;
}

__global__ void hlrb_split_kernel(int C, int D, int Dp, const float* __restrict__ theta, int ldt,
                                  __nv_bfloat16* __restrict__ t3) {
  const int c = blockIdx.y;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < Dp; d += gridDim.x * blockDim.x)
    split_elem(c, d, D, Dp, theta, ldt, t3);
}

// X [N][ldx] -> Xt [Np/64][D][64], zero for n >= N.  32x32 tiles through
// shared memory.
__global__ void hlrb_transpose_kernel(int N, int D, int Np, const __nv_bfloat16* __restrict__ X, int ldx,
                                      __nv_bfloat16* __restrict__ Xt) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int n0 = blockIdx.x * 32, d0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
  for (int j = ty; j < 32; j += 8) {
    const int n = n0 + j, d = d0 + tx;
    tile[j][tx] = (n < N && d < D) ? X[(size_t)n * ldx + d] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const int d = d0 + j, n = n0 + tx;
    if (d < D && n < Np) Xt[((size_t)(n >> 6) * D + d) * 64 + (n & 63)] = tile[tx][j];
  }
}

// Forward epilogue: rows are chains, columns are data rows.  LL: sum the
// log-likelihood terms; R: write the residual parts for the backward pass
// (a leapfrog step that only needs the gradient skips the LL work).
//
// With s = 2y - 1 and u = s t, the Bernoulli-logit term and residual are
//   y t - softplus(t) = min(u, 0) - log(1 + e),   e = exp(-|t|),
//   y - sigmoid(t)    = s * (u >= 0 ? e : 1) / (1 + e),
// one MUFU exp2, log2 and reciprocal each (hardware exp2 / log2: the
// absolute log-density error at N = 2e6 is 0.037 nats, 4e-8 relative, and
// its chain-to-chain differences - what an accept test sees - are 0.004).
// The 32 terms of a column chunk are summed in four interleaved FP32
// partials (min(u, 0) and log2(1 + e) kept apart; both parts of a term
// have the same sign, so nothing cancels), and the chunk sums go into a
// Kahan-compensated running sum per chain and column group.  Rows at or
// past N carry s = 0: no term, zero residual.
// The hardware approximations (one MUFU operation each, subnormals flushed):
// 2^x, log2 x and 1/x.
__device__ __forceinline__ float ex2_ftz(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float lg2_ftz(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// One chunk of NW columns of the forward epilogue for one chain: t = v[i] at
// rows with s = sv[i] (2y - 1, or 0 past N; FULL: no such rows), residual
// into rv, the chunk's log-likelihood terms added to the Kahan pair
// (acc, comp).
template <bool LL, bool R, bool FULL, int NW = 32>
__device__ __forceinline__ void ll_resid_chunk(const float* v, const float* sv, float* rv, float& acc, float& comp) {
  float s1[4] = {0.0f, 0.0f, 0.0f, 0.0f}, s2[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int i = 0; i < NW; ++i) {
    const float t = v[i], sg = sv[i];
    const float u = sg * t;
    const float e = ex2_ftz(-1.4426950408889634f * fabsf(t));   // exp(-|t|), 0 below 2^-126
    const float ope = 1.0f + e;                                  // in [1, 2]
    if (LL) {
      s1[i & 3] += fminf(u, 0.0f);
      const float l2 = lg2_ftz(ope);
      s2[i & 3] += (FULL || sg != 0.0f) ? l2 : 0.0f;
    }
    if (R) {
      const float inv = rcp_ftz(ope);
      rv[i] = sg * (u >= 0.0f ? e * inv : inv);
    }
  }
  if (LL) {
    const float part = ((s1[0] + s1[1]) + (s1[2] + s1[3])) -
                       0.69314718055994531f * ((s2[0] + s2[1]) + (s2[2] + s2[3]));
    const float yk = part - comp;   // Kahan-compensated running sum
    const float tk = acc + yk;
    comp = (tk - acc) - yk;
    acc = tk;
  }
}

// hi = bf16(r), mid = bf16(r - hi) of two values, each pair packed in one
// 32-bit word (the difference r - hi is exact in FP32).
__device__ __forceinline__ void split_pair(float r0, float r1, uint32_t& hi, uint32_t& mid) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(r0, r1);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  const float h0 = __uint_as_float(hi << 16), h1 = __uint_as_float(hi & 0xffff0000u);
  const __nv_bfloat162 m = __floats2bfloat162_rn(r0 - h0, r1 - h1);
  mid = *reinterpret_cast<const uint32_t*>(&m);
}

template <bool LL, bool R, int W, int BN>
struct FwdEpi {
  static constexpr int kSmem = BN * 4;
  static constexpr int kWarps = W;
  static constexpr int kGroups = W / 4;
  const int* y;
  __nv_bfloat16* r3;   // NULL: log density only
  float* llpart;       // [fwd_tiles][kGroups][C]
  int N, Np, C;
  // per-thread state
  const float* ss;     // s = 2y - 1 of the tile's rows (0 past N), shared memory
  int n0;
  float acc, comp;

  __device__ void begin(int, int nt, int, char* smem, int etid) {
    float* s = reinterpret_cast<float*>(smem);
    n0 = nt * BN;
    for (int j = etid; j < BN; j += 32 * W) {
      const int n = n0 + j;
      s[j] = n < N ? (y[n] ? 1.0f : -1.0f) : 0.0f;
    }
    ss = s;
    acc = 0.0f;
    comp = 0.0f;
  }

  __device__ void rows(int c, int col0, const float* v, bool ok) {
    if (!ok) return;
    float rv[32], sv[32];
    const float4* s4 = reinterpret_cast<const float4*>(ss + (col0 - n0));
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 a = s4[q];
      sv[4 * q] = a.x;
      sv[4 * q + 1] = a.y;
      sv[4 * q + 2] = a.z;
      sv[4 * q + 3] = a.w;
    }
    if (col0 + 32 <= N) ll_resid_chunk<LL, R, true>(v, sv, rv, acc, comp);   // uniform over the warp
    else ll_resid_chunk<LL, R, false>(v, sv, rv, acc, comp);
    if (R && col0 < Np) {
      // K-blocked [Np/64][2][C][64]: part p of chain c for rows col0..col0+31;
      // hi = bf16(r), mid = bf16(r - hi) (the difference is exact in FP32),
      // converted two at a time
      __nv_bfloat16* base = r3 + ((size_t)(col0 >> 6) * R_PARTS * C + c) * 64 + (col0 & 63);
      uint32_t ph[16], pm[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) split_pair(rv[2 * i], rv[2 * i + 1], ph[i], pm[i]);
      uint4* dh = reinterpret_cast<uint4*>(base);
      uint4* dm = reinterpret_cast<uint4*>(base + (size_t)C * 64);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        dh[i] = make_uint4(ph[4 * i], ph[4 * i + 1], ph[4 * i + 2], ph[4 * i + 3]);
        dm[i] = make_uint4(pm[4 * i], pm[4 * i + 1], pm[4 * i + 2], pm[4 * i + 3]);
      }
    }
  }

  __device__ void end(int, int nt, int, int c, bool ok, int cg) {
    if (LL && ok) llpart[((size_t)nt * kGroups + cg) * C + c] = acc;
  }
};

// Backward epilogue: rows are chains, columns are features; one FP32 partial
// tile per split.
struct GradEpi {
  static constexpr int kSmem = 0;
  static constexpr int kWarps = 4;
  float* w;   // [splits][C][ldw]
  int C, D, ldw;
  int sp;
  __device__ void begin(int, int, int split, char*, int) { sp = split; }
  __device__ void rows(int c, int col0, const float* v, bool ok) {
    if (!ok || col0 >= D) return;
    float* out = w + ((size_t)sp * C + c) * ldw + col0;
    if (col0 + 32 <= ldw) {
      float4* o4 = reinterpret_cast<float4*>(out);
#pragma unroll
      for (int i = 0; i < 8; ++i) o4[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
  }
  __device__ void end(int, int, int, int, bool, int) {}
};

__device__ __forceinline__ void prior_term(int kind, double a, double b, double x, double& ll, double& g) {
  if (kind == AB_PRIOR_NORMAL) {
    // Normal(0, a): log density and derivative
    ll = -0.5 * log(2.0 * M_PI * a) - 0.5 * x * x / a;
    g = -x / a;
  } else {
    // Student-t(nu = a, scale = b)
    const double nu = a, z = x / b;
    ll = lgamma(0.5 * (nu + 1.0)) - lgamma(0.5 * nu) - 0.5 * log(nu * M_PI) - log(b) -
         0.5 * (nu + 1.0) * log1p(z * z / nu);
    g = -(nu + 1.0) * x / (nu * b * b + x * x);
  }
}

// One block per chain: logp[c] (FP64) and grad[c][0..D-1] (FP32) from the
// partials, in a fixed order; either output may be NULL.
__device__ __forceinline__ void finish_chain(int c, int C, int D, int fwd_tiles, int splits, int ldw,
                                             const float* __restrict__ llpart, const float* __restrict__ w,
                                             const float* __restrict__ theta, int ldt, int prior, double pa,
                                             double pb, double* __restrict__ logp, float* __restrict__ grad,
                                             int ldg) {
  __shared__ double red[33];
  double s = 0.0;
  if (logp)
    for (int t = threadIdx.x; t < fwd_tiles; t += blockDim.x) s += (double)llpart[(size_t)t * C + c];
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    double pl, pg;
    prior_term(prior, pa, pb, (double)theta[(size_t)c * ldt + d], pl, pg);
    s += pl;
    if (grad) {
      double g = pg;
      for (int k = 0; k < splits; ++k) g += (double)w[((size_t)k * C + c) * ldw + d];
      grad[(size_t)c * ldg + d] = (float)g;
    }
  }
  s = block_sum_f64(s, red);
  if (logp && threadIdx.x == 0) logp[c] = s;
}

__global__ void __launch_bounds__(256) hlrb_finish_kernel(int C, int D, int fwd_tiles, int splits, int ldw,
                                                          const float* __restrict__ llpart,
                                                          const float* __restrict__ w, const float* __restrict__ theta,
                                                          int ldt, int prior, double pa, double pb,
                                                          double* __restrict__ logp, float* __restrict__ grad,
                                                          int ldg) {
  finish_chain(blockIdx.x, C, D, fwd_tiles, splits, ldw, llpart, w, theta, ldt, prior, pa, pb, logp, grad, ldg);
}

}  // namespace

template <int W, int BN>
int launch_forward(const ab_hlrb_model* m, const CUtensorMap& ma, const CUtensorMap& mb, const tc::Shape& fs,
                   bool logp, bool grad, __nv_bfloat16* r3, float* llp, int Np, int C, int* err, cudaStream_t st) {
  if (logp && grad) {
    FwdEpi<true, true, W, BN> fe{m->y, r3, llp, m->N, Np, C, nullptr, 0, 0.0f, 0.0f};
    return tc::launch_gemm<BN, 3, 1>(ma, mb, fs, fe, err, st);
  }
  if (logp) {
    FwdEpi<true, false, W, BN> fe{m->y, r3, llp, m->N, Np, C, nullptr, 0, 0.0f, 0.0f};
    return tc::launch_gemm<BN, 3, 1>(ma, mb, fs, fe, err, st);
  }
  FwdEpi<false, true, W, BN> fe{m->y, r3, llp, m->N, Np, C, nullptr, 0, 0.0f, 0.0f};
  return tc::launch_gemm<BN, 3, 1>(ma, mb, fs, fe, err, st);
}

template <int BN>
int launch_forward_w(int groups, const ab_hlrb_model* m, const CUtensorMap& ma, const CUtensorMap& mb,
                     const tc::Shape& fs, bool logp, bool grad, __nv_bfloat16* r3, float* llp, int Np, int C,
                     int* err, cudaStream_t st) {
  if (groups == 1) return launch_forward<4, BN>(m, ma, mb, fs, logp, grad, r3, llp, Np, C, err, st);
  if (groups == 2) return launch_forward<8, BN>(m, ma, mb, fs, logp, grad, r3, llp, Np, C, err, st);
  return launch_forward<16, BN>(m, ma, mb, fs, logp, grad, r3, llp, Np, C, err, st);
}

int hlrb_logp_grad(const ab_hlrb_model* m, int C, const float* theta, int ldt, double* logp, float* grad, int ldg,
                   const ab_hlrb_config* cfg, void* work, int* err, cudaStream_t st) {
  const int N = m->N, D = m->D;
  const Layout L = layout(N, D, C, cfg);
  char* wb = static_cast<char*>(work);
  __nv_bfloat16* t3 = reinterpret_cast<__nv_bfloat16*>(wb + L.off_t3);
  __nv_bfloat16* r3 = reinterpret_cast<__nv_bfloat16*>(wb + L.off_r3);
  float* llp = reinterpret_cast<float*>(wb + L.off_ll);
  float* w = reinterpret_cast<float*>(wb + L.off_w);

  hlrb_split_kernel<<<dim3(ceil_div(L.Dp, 256), C), 256, 0, st>>>(C, D, L.Dp, theta, ldt, t3);
  AB_LAUNCH_CHECK("hlrb_split_kernel");

  int rc;
  CUtensorMap ma, mb;
  if ((rc = tc::encode_2d_bf16(&ma, t3, C, 3 * L.Dp, 3 * L.Dp, tc::BM))) return rc;
  if ((rc = tc::encode_2d_bf16(&mb, m->X, N, D, m->ldx, L.fwd_bn))) return rc;
  const tc::Shape fs = tc::make_shape(C, N, D, 1, tc::row_major(L.Dp), tc::row_major(0), L.fwd_bn);
  rc = L.fwd_bn == 128
           ? launch_forward_w<128>(L.groups, m, ma, mb, fs, logp != nullptr, grad != nullptr, r3, llp, L.Np, C, err, st)
           : launch_forward_w<256>(L.groups, m, ma, mb, fs, logp != nullptr, grad != nullptr, r3, llp, L.Np, C, err, st);
  if (rc) return rc;

  if (grad) {
    const int nb = L.Np / 64;
    if ((rc = tc::encode_2d_bf16(&ma, r3, (uint64_t)nb * R_PARTS * C, 64, 64, tc::BM))) return rc;
    const int bn = L.bn;
    if ((rc = tc::encode_2d_bf16(&mb, m->Xt, (uint64_t)nb * D, 64, 64, bn))) return rc;
    GradEpi ge{w, C, D, L.ldw, 0};
    const tc::Shape bs = tc::make_shape(C, D, N, L.splits, tc::k_blocked(R_PARTS, C), tc::k_blocked(1, D), bn);
    AB_REQUIRE(bs.splits == L.splits, AB_ERR_STATE, "hlrb: split arithmetic mismatch");
    if (bn == 32) rc = tc::launch_gemm<32, R_PARTS, 1>(ma, mb, bs, ge, err, st);
    else if (bn == 64) rc = tc::launch_gemm<64, R_PARTS, 1>(ma, mb, bs, ge, err, st);
    else rc = tc::launch_gemm<128, R_PARTS, 1>(ma, mb, bs, ge, err, st);
    if (rc) return rc;
  }
  hlrb_finish_kernel<<<C, 256, 0, st>>>(C, D, L.fwd_tiles * L.groups, L.splits, L.ldw, llp, w, theta, ldt, m->prior,
                                        m->prior_a, m->prior_b, logp, grad, ldg);
  AB_LAUNCH_CHECK("hlrb_finish_kernel");
  return AB_OK;
}

int hlrb_check_model(const ab_hlrb_model* m) {
  AB_REQUIRE(m, AB_ERR_ARG, "hlrb: null model");
  AB_REQUIRE(m->N > 0 && m->D > 0 && m->D <= 65536, AB_ERR_ARG, "hlrb: bad sizes N=%d D=%d", m->N, m->D);
  AB_REQUIRE(m->X && m->Xt && m->y, AB_ERR_ARG, "hlrb: null data pointer");
  AB_REQUIRE(m->ldx >= m->D && m->ldx % 8 == 0, AB_ERR_ARG, "hlrb: ldx must be >= D and a multiple of 8");
  AB_REQUIRE(m->prior == AB_PRIOR_NORMAL || m->prior == AB_PRIOR_STUDENT_T, AB_ERR_ARG, "hlrb: unknown prior");
  AB_REQUIRE(m->prior_a > 0.0 && (m->prior == AB_PRIOR_NORMAL || m->prior_b > 0.0), AB_ERR_ARG,
             "hlrb: prior parameters must be positive");
  return AB_OK;
}

size_t hlrb_workspace_bytes(int N, int D, int C, const ab_hlrb_config* cfg) { return layout(N, D, C, cfg).total; }

}  // namespace ab

using namespace ab;

extern "C" size_t ab_hlrb_xt_elems(int N, int D) {
  if (N <= 0 || D <= 0) return 0;
  return (size_t)D * (size_t)((N + 63) / 64 * 64);
}

extern "C" int ab_hlrb_transpose(int N, int D, const void* X, int ldx, void* Xt, void* stream) {
  AB_REQUIRE(N > 0 && D > 0 && ldx >= D, AB_ERR_ARG, "ab_hlrb_transpose: bad sizes");
  AB_REQUIRE(X && Xt, AB_ERR_ARG, "ab_hlrb_transpose: null pointer");
  const int Np = (N + 63) / 64 * 64;
  hlrb_transpose_kernel<<<dim3(ceil_div(Np, 32), ceil_div(D, 32)), dim3(32, 8), 0, as_stream(stream)>>>(
      N, D, Np, static_cast<const __nv_bfloat16*>(X), ldx, static_cast<__nv_bfloat16*>(Xt));
  AB_LAUNCH_CHECK("hlrb_transpose_kernel");
  return AB_OK;
}

extern "C" size_t ab_hlrb_workspace_bytes(int N, int D, int C) {
  if (N <= 0 || D <= 0 || C <= 0) return 0;
  return hlrb_workspace_bytes(N, D, C, nullptr);
}

extern "C" size_t ab_hlrb_workspace_bytes_cfg(int N, int D, int C, const ab_hlrb_config* cfg) {
  if (N <= 0 || D <= 0 || C <= 0 || check_config(cfg)) return 0;
  return hlrb_workspace_bytes(N, D, C, cfg);
}

extern "C" int ab_hlrb_logp_grad_cfg(const ab_hlrb_model* m, int C, const float* theta, int ldt, double* logp,
                                     float* grad, int ldg, const ab_hlrb_config* cfg, void* work, int* err,
                                     void* stream) {
  int rc = hlrb_check_model(m);
  if (rc) return rc;
  if ((rc = check_config(cfg))) return rc;
  AB_REQUIRE(C > 0 && C <= 65535, AB_ERR_ARG, "ab_hlrb_logp_grad: C must be 1..65535");
  AB_REQUIRE(theta && work && (logp || grad), AB_ERR_ARG, "ab_hlrb_logp_grad: null pointer");
  AB_REQUIRE(ldt >= m->D && (!grad || ldg >= m->D), AB_ERR_ARG, "ab_hlrb_logp_grad: leading dimension too small");
  AB_REQUIRE((reinterpret_cast<uintptr_t>(work) & 255) == 0, AB_ERR_ARG, "ab_hlrb_logp_grad: workspace must be 256-byte aligned");
  return hlrb_logp_grad(m, C, theta, ldt, logp, grad, ldg, cfg, work, err, as_stream(stream));
}

extern "C" int ab_hlrb_logp_grad(const ab_hlrb_model* m, int C, const float* theta, int ldt, double* logp,
                                 float* grad, int ldg, void* work, int* err, void* stream) {
  return ab_hlrb_logp_grad_cfg(m, C, theta, ldt, logp, grad, ldg, nullptr, work, err, stream);
}

// ---- grouped pass: many instances, one launch per stage ---------------------
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

namespace ab {
namespace {

using GFwd = FwdEpi<true, true, 8, 256>;   // the built-in forward shape, logp and gradient
constexpr int G_BWD_BN = 128;              // widest backward tile; each instance uses its own bwd_bn(D)

struct GSplit {
  const float* theta;
  __nv_bfloat16* t3;
  int ldt, C, D, Dp;
};

struct GFinish {
  const float* llpart;
  const float* w;
  const float* theta;
  double* logp;
  float* grad;
  double pa, pb;
  int C, D, fwd_parts, splits, ldw, ldt, prior, ldg;
};

// The launch header: problems in use and tiles of the forward and backward
// GEMMs (the split and finish kernels read n from the forward's).
struct GHeads {
  tc::GHead fwd, bwd;
};

__global__ void hlrg_split_kernel(const GSplit* __restrict__ tab, const GHeads* __restrict__ head) {
  if ((int)blockIdx.z >= head->fwd.n) return;
  const GSplit q = tab[blockIdx.z];
  const int c = blockIdx.y;
  if (c >= q.C) return;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < q.Dp; d += gridDim.x * blockDim.x)
    split_elem(c, d, q.D, q.Dp, q.theta, q.ldt, q.t3);
}

__global__ void __launch_bounds__(256) hlrg_finish_kernel(const GFinish* __restrict__ tab,
                                                          const GHeads* __restrict__ head) {
  if ((int)blockIdx.y >= head->fwd.n) return;
  const GFinish q = tab[blockIdx.y];
  if ((int)blockIdx.x >= q.C) return;
  finish_chain(blockIdx.x, q.C, q.D, q.fwd_parts, q.splits, q.ldw, q.llpart, q.w, q.theta, q.ldt, q.prior, q.pa, q.pb,
               q.logp, q.grad, q.ldg);
}

struct HlrgInst {
  ab_hlrb_model m;
  int C;
  Layout L;          // unfused pass: the built-in launch shape
  char* work;
  tc::GProblem fwd, bwd;
  GFwd fe;
  GradEpi ge;
  // fused pass (every instance D <= 256): theta parts, partial sums, maps
  int Dp = 0, Dn = 0, rtiles = 0, nseg = 0;
  size_t f_t3 = 0, f_llp = 0, f_gw = 0, f_total = 0;
  const float* theta = nullptr;
  double* logp = nullptr;
  float* grad = nullptr;
  int ldt = 0, ldg = 0;
};

inline size_t al256(size_t a) { return (a + 255) & ~size_t(255); }

// ---- fused pass (D <= 256): forward, residual and backward in one kernel ----
//
// One persistent CTA per SM walks a list of work units; a unit is one
// instance's chain tile (128 chains) over a segment of up to F_SEG_TILES
// row tiles of 128 data rows.  Per row tile:
//   forward   T[128 chains x 128 rows] = Theta3 . X_tile^T into one of two
//             tensor-memory accumulators (3 bf16 parts of theta, K = D);
//   epilogue  log-likelihood terms (Kahan sum per chain over the unit) and
//             the residual r = y - sigmoid(t) as two bf16 parts, written to
//             shared memory in the 128-byte-swizzled K-major layout the MMA
//             reads (no global scratch);
//   backward  G[128 chains x Dn] += R_p . Xt_block^T, the transposed X block
//             [D rows x 64] fetched by TMA from the K-blocked copy of X; G
//             stays in tensor memory (columns 256..511) for the whole unit.
// The MMA issue order F(0) F(1) B(0) F(2) B(1) ... B(n-1) lets the forward
// of the next row tile run while the epilogue works on the current one.  At
// the end of a unit the epilogue writes the unit's partial log likelihood
// [seg][2 column groups][C] and gradient [seg][C][Dn]; the finishing kernel
// adds the segments in a fixed order.  A unit's results depend only on its
// instance and rows, never on which CTA ran it or what else is in the
// launch, so a group of instances gives each instance the numbers it gets
// alone.  Roles: warp 0 lane 0 TMA producer, warp 1 lane 0 MMA issuer,
// warps 2..17 epilogue (column group g = 32 columns, taken 16 at a time;
// lane quarter = warp % 4).  Every wait is bounded as in gemm_kernel.
constexpr int F_ROWS = 128;
constexpr int F_SEG_TILES = 64;                            // row tiles per unit (8192 rows)
constexpr int F_MAX_D = 256;
constexpr int F_EPI_WARPS = 16;
constexpr int F_GROUPS = F_EPI_WARPS / 4;                 // column groups of 32
constexpr int F_THREADS = 64 + 32 * F_EPI_WARPS;
constexpr int F_STAGES = 2;
constexpr int F_A_BYTES = 128 * 64 * 2;                    // one 128 x 64 bf16 box
constexpr int F_STAGE_BYTES = 3 * F_A_BYTES + F_ROWS * 128; // theta parts + X tile; an Xt block uses Dn * 128
constexpr int F_ROFF = F_STAGES * F_STAGE_BYTES;           // residual parts: [2 parts][2 K-blocks] boxes
constexpr int F_YOFF = F_ROFF + 4 * F_A_BYTES;             // s values [2][128] f32
constexpr int F_BAROFF = F_YOFF + 2 * F_ROWS * 4;
constexpr int F_SMEM = F_BAROFF + 256 + 1024;
constexpr int F_TMEM_COLS = 512;                           // T0 | T1 | G
static_assert(F_SMEM <= tc::SMEM_BUDGET, "fused pass exceeds shared memory");

struct alignas(64) FInst {
  CUtensorMap t3, x, xt;
  const int* y;
  float* llp;   // [nseg][F_GROUPS][C]
  float* gw;    // [nseg][C][Dn]
  int N, D, Dp, Dn, C;
};

struct FUnit {
  int inst, m, r0, r1, seg;
};

__global__ void __launch_bounds__(F_THREADS, 1)
hlrf_kernel(const FInst* __restrict__ insts, const FUnit* __restrict__ units, const int* __restrict__ cta_off,
            int* __restrict__ err) {
  using namespace tc;
  const int u_beg = cta_off[blockIdx.x], u_end = cta_off[blockIdx.x + 1];
  if (u_beg >= u_end) return;   // uniform over the CTA
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* ring = base;
  unsigned char* rbuf = base + F_ROFF;
  float* ys = reinterpret_cast<float*>(base + F_YOFF);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + F_BAROFF);
  uint64_t* empty = full + F_STAGES;
  uint64_t* acc_full = empty + F_STAGES;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* r_full = acc_empty + 2;
  uint64_t* r_empty = r_full + 1;
  uint64_t* g_full = r_empty + 1;
  uint64_t* g_empty = g_full + 1;
  uint64_t* drain = g_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);
  int* epi_fail = fail + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < F_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int b = 0; b < 2; ++b) { mbar_init(&acc_full[b], 1); mbar_init(&acc_empty[b], F_EPI_WARPS); }
    mbar_init(r_full, F_EPI_WARPS);
    mbar_init(r_empty, 1);
    mbar_init(g_full, 1);
    mbar_init(g_empty, F_EPI_WARPS);
    mbar_init(drain, 1);
    *fail = 0;
    *epi_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)F_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  int issued = 0;
  if (warp == 0) {
    if (lane == 0) {
      int g = 0, last = -1;
      for (int u = u_beg; u < u_end && !*(volatile int*)fail; ++u) {
        const FUnit U = units[u];
        const FInst* I = insts + U.inst;
        if (U.inst != last) {
          tensormap_acquire(&I->t3);
          tensormap_acquire(&I->x);
          tensormap_acquire(&I->xt);
          last = U.inst;
        }
        const int n = U.r1 - U.r0, ksteps = I->Dp / BK, D = I->D, Dp = I->Dp;
        const uint32_t bbytes = (uint32_t)(I->Dn * 128);
        bool bad = false;
        for (int k = 0; k <= n && !bad; ++k) {
          if (k < n) {
            for (int kb = 0; kb < ksteps; ++kb, ++g) {
              const int s = g % F_STAGES;
              if (g >= F_STAGES && !mbar_wait(&empty[s], ((g / F_STAGES) & 1) ^ 1)) { *fail = 1; bad = true; break; }
              if (*(volatile int*)fail) { bad = true; break; }
              unsigned char* a = ring + s * F_STAGE_BYTES;
              mbar_expect_tx(&full[s], (uint32_t)F_STAGE_BYTES);
#pragma unroll
              for (int p = 0; p < 3; ++p) tma_load_2d(a + p * F_A_BYTES, &I->t3, &full[s], kb * BK + p * Dp, U.m * BM);
              tma_load_2d(a + 3 * F_A_BYTES, &I->x, &full[s], kb * BK, (U.r0 + k) * F_ROWS);
              ++issued;
            }
          }
          if (k >= 1 && !bad) {
            for (int j = 0; j < 2; ++j, ++g) {
              const int s = g % F_STAGES;
              if (g >= F_STAGES && !mbar_wait(&empty[s], ((g / F_STAGES) & 1) ^ 1)) { *fail = 1; bad = true; break; }
              if (*(volatile int*)fail) { bad = true; break; }
              unsigned char* a = ring + s * F_STAGE_BYTES;
              mbar_expect_tx(&full[s], bbytes);
              tma_load_2d(a, &I->xt, &full[s], 0, (2 * (U.r0 + k - 1) + j) * D);
              ++issued;
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc_t = make_idesc(F_ROWS);
      int g = 0, it = 0, rb = 0, gu = 0;
      bool bad = false;
      for (int u = u_beg; u < u_end && !bad; ++u) {
        const FUnit U = units[u];
        const FInst* I = insts + U.inst;
        const int n = U.r1 - U.r0, ksteps = I->Dp / BK;
        const uint32_t idesc_g = make_idesc(I->Dn);
        for (int k = 0; k <= n && !bad; ++k) {
          if (k < n) {
            const int buf = it & 1;
            if (it >= 2 && !mbar_wait(&acc_empty[buf], ((it >> 1) - 1) & 1)) { *fail = 1; bad = true; break; }
            if (*(volatile int*)fail) { bad = true; break; }
            fence_after();
            const uint32_t d = tmem + (uint32_t)(buf * F_ROWS);
            for (int kb = 0; kb < ksteps; ++kb, ++g) {
              const int s = g % F_STAGES;
              if (!mbar_wait(&full[s], (g / F_STAGES) & 1)) { *fail = 1; bad = true; break; }
              if (*(volatile int*)fail) { bad = true; break; }
              fence_after();
              unsigned char* a = ring + s * F_STAGE_BYTES;
#pragma unroll
              for (int kk = 0; kk < BK / 16; ++kk)
#pragma unroll
                for (int p = 0; p < 3; ++p)
                  mma_bf16(d, make_desc(a + p * F_A_BYTES) + 2 * kk, make_desc(a + 3 * F_A_BYTES) + 2 * kk, idesc_t,
                           (kb > 0 || kk > 0 || p > 0) ? 1u : 0u);
              mma_commit(&empty[s]);
            }
            if (bad) break;
            mma_commit(&acc_full[buf]);
            ++it;
          }
          if (k >= 1) {
            if (!mbar_wait(r_full, rb & 1)) { *fail = 1; bad = true; break; }
            if (k == 1 && gu >= 1 && !mbar_wait(g_empty, (gu - 1) & 1)) { *fail = 1; bad = true; break; }
            if (*(volatile int*)fail) { bad = true; break; }
            fence_after();
            const uint32_t dg = tmem + 2u * F_ROWS;
            for (int j = 0; j < 2; ++j, ++g) {
              const int s = g % F_STAGES;
              if (!mbar_wait(&full[s], (g / F_STAGES) & 1)) { *fail = 1; bad = true; break; }
              if (*(volatile int*)fail) { bad = true; break; }
              fence_after();
              unsigned char* b = ring + s * F_STAGE_BYTES;
#pragma unroll
              for (int kk = 0; kk < BK / 16; ++kk)
#pragma unroll
                for (int p = 0; p < 2; ++p)
                  mma_bf16(dg, make_desc(rbuf + (p * 2 + j) * F_A_BYTES) + 2 * kk, make_desc(b) + 2 * kk, idesc_g,
                           (k > 1 || j > 0 || kk > 0 || p > 0) ? 1u : 0u);
              mma_commit(&empty[s]);
            }
            if (bad) break;
            mma_commit(r_empty);
            ++rb;
          }
        }
        if (bad) break;
        mma_commit(g_full);
        ++gu;
      }
      mma_commit(drain);
      if (!mbar_wait(drain, 0)) *fail = 1;
    }
  } else {
    const int qw = warp & 3;                 // TMEM lane quarter
    const int grp = (warp - 2) >> 2;         // column group: columns [32 grp, 32 grp + 32)
    const int etid = (warp - 2) * 32 + lane;
    const int cl = qw * 32 + lane;           // chain within the tile
    const uint32_t lane_base = tmem + ((uint32_t)(qw * 32) << 16);
    int it = 0, gu = 0;
    bool bad = false;   // this thread's failure so far (uniform over the warp)
    // y of row etid of the next tile, loaded one tile ahead (threads etid < 128)
    int pf_y = 0;
    bool pf_v = false;
    auto prefetch = [&](int uu, int kk) {
      if (etid < F_ROWS && uu < u_end) {
        const FUnit V = units[uu];
        const FInst* J = insts + V.inst;
        const int nn = (V.r0 + kk) * F_ROWS + etid;
        pf_v = nn < J->N;
        pf_y = pf_v ? J->y[nn] : 0;
      }
    };
    prefetch(u_beg, 0);
    for (int u = u_beg; u < u_end; ++u) {
      const FUnit U = units[u];
      const FInst* I = insts + U.inst;
      const int n = U.r1 - U.r0, N = I->N, C = I->C, Dn = I->Dn;
      const int chain = U.m * BM + cl;
      const bool ok = chain < C;
      float acc = 0.0f, comp = 0.0f;
      bool stop = false;
      for (int k = 0; k < n; ++k) {
        const int buf = it & 1;
        const int row0 = (U.r0 + k) * F_ROWS;
        if (etid < F_ROWS) ys[buf * F_ROWS + etid] = pf_v ? (pf_y ? 1.0f : -1.0f) : 0.0f;
        if (k + 1 < n) prefetch(u, k + 1);
        else prefetch(u + 1, 0);
        // the barrier ORs every epilogue thread's failure flag: all stop together
        if (epi_sync_or(32 * F_EPI_WARPS, bad)) { stop = true; break; }
        bool okw = __all_sync(0xffffffffu, mbar_wait(&acc_full[buf], (it >> 1) & 1));
        if (it >= 1) okw = __all_sync(0xffffffffu, okw && mbar_wait(r_empty, (it - 1) & 1));
        fence_after();
        const bool have = __all_sync(0xffffffffu, okw && !*(volatile int*)fail);
        const uint32_t tcol = (uint32_t)(buf * F_ROWS + grp * 32);
        const float* sv0 = ys + buf * F_ROWS + grp * 32;
        // the group's 32 columns lie in residual K-block grp / 2, 16-byte
        // chunks 4 (grp % 2) .. +3 of each chain row
        unsigned char* rowh = rbuf + (0 * 2 + (grp >> 1)) * F_A_BYTES + cl * 128;
        unsigned char* rowm = rbuf + (1 * 2 + (grp >> 1)) * F_A_BYTES + cl * 128;
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          float v[16], sv[16], rv[16];
          if (have) {
            uint32_t r[16];
            tmem_ld16_issue(lane_base + tcol + cc * 16, r);
            tmem_wait16(r);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
          } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = 0.0f;
          }
          const float4* s4 = reinterpret_cast<const float4*>(sv0 + cc * 16);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float4 a = s4[i];
            sv[4 * i] = a.x;
            sv[4 * i + 1] = a.y;
            sv[4 * i + 2] = a.z;
            sv[4 * i + 3] = a.w;
          }
          if (row0 + grp * 32 + cc * 16 + 16 <= N) ll_resid_chunk<true, true, true, 16>(v, sv, rv, acc, comp);
          else ll_resid_chunk<true, true, false, 16>(v, sv, rv, acc, comp);
          // residual parts into the swizzled K-major boxes: chain row cl,
          // 16-byte chunk c16 of the row stored at c16 ^ (cl & 7)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            uint32_t h[4], m[4];
#pragma unroll
            for (int e2 = 0; e2 < 4; ++e2) split_pair(rv[8 * q + 2 * e2], rv[8 * q + 2 * e2 + 1], h[e2], m[e2]);
            const int c16 = ((grp & 1) * 4 + cc * 2 + q) ^ (cl & 7);
            *reinterpret_cast<uint4*>(rowh + c16 * 16) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4*>(rowm + c16 * 16) = make_uint4(m[0], m[1], m[2], m[3]);
          }
        }
        fence_before();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // residual writes -> tensor core
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&acc_empty[buf]);
          mbar_arrive(r_full);
        }
        if (!have) bad = true;
        ++it;
      }
      if (stop) break;
      if (ok) I->llp[((size_t)U.seg * F_GROUPS + grp) * C + chain] = acc;
      // the unit's gradient: columns [64 grp, 64 grp + 64) of G
      const bool okg = __all_sync(0xffffffffu, mbar_wait(g_full, gu & 1) && !*(volatile int*)fail);
      fence_after();
      const int c_end = min(Dn, grp * 64 + 64);
      for (int c0 = grp * 64; c0 < c_end; c0 += 32) {
        if (!okg) break;
        uint32_t r[32];
        tmem_ld32_issue(lane_base + 2u * F_ROWS + (uint32_t)c0, r);
        tmem_wait32(r);
        if (ok) {
          float4* o = reinterpret_cast<float4*>(I->gw + ((size_t)U.seg * C + chain) * Dn + c0);
          const int lim = min(32, Dn - c0);   // Dn is a multiple of 16
#pragma unroll
          for (int i = 0; i < 8; ++i)
            if (4 * i < lim)
              o[i] = make_float4(__uint_as_float(r[4 * i]), __uint_as_float(r[4 * i + 1]), __uint_as_float(r[4 * i + 2]),
                                 __uint_as_float(r[4 * i + 3]));
        }
      }
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(g_empty);
      if (!okg) bad = true;
      ++gu;
    }
    if (bad) *(volatile int*)epi_fail = 1;
  }
  __syncwarp();
  if (threadIdx.x == 0 && *(volatile int*)fail) {
    for (int g = max(0, issued - F_STAGES); g < issued; ++g) mbar_wait(&full[g % F_STAGES], (g / F_STAGES) & 1);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)F_TMEM_COLS)
                 : "memory");
  }
  if (threadIdx.x == 0 && (*(volatile int*)fail || *(volatile int*)epi_fail) && err) atomicExch(err, AB_ERR_TIMEOUT);
}

}  // namespace
}  // namespace ab

struct ab_hlrg {
  std::vector<ab::HlrgInst> inst;
  std::vector<ab::FInst> finst;   // fused pass: per instance (maps, pointers, sizes)
  bool fused = false;             // every instance has D <= 256: one fused kernel per pass
  int C_max = 0, Dp_max = 0, grid_fwd = 0, grid_bwd = 0, grid_f = 0, n_active = 0, units_max = 0;
  bool ready = false;
  char* work = nullptr;    // every instance's workspace
  char* tab = nullptr;     // device tables
  size_t o_fwd = 0, o_bwd = 0, o_fe = 0, o_ge = 0, o_sp = 0, o_fin = 0, o_fi = 0, o_fu = 0, o_off = 0, bytes = 0;
  unsigned char* stage = nullptr;   // host copy of the tables (256-byte aligned)
  ~ab_hlrg() {
    std::free(stage);
    cudaFree(work);
    cudaFree(tab);
  }
};

namespace ab {
namespace {
// Fused pass: the work units of one instance (chain tile, row segment).
void fused_units(const HlrgInst& q, int inst, std::vector<FUnit>& out) {
  const int mt = (q.C + tc::BM - 1) / tc::BM;
  for (int m = 0; m < mt; ++m)
    for (int sg = 0; sg < q.nseg; ++sg)
      out.push_back(FUnit{inst, m, sg * F_SEG_TILES, std::min(q.rtiles, (sg + 1) * F_SEG_TILES), sg});
}

// Longest-processing-time-first assignment of units to CTAs; writes the
// units grouped by CTA and the CTA offsets.
void assign_units(const std::vector<FUnit>& u, const std::vector<HlrgInst>& inst, const std::vector<int>& act,
                  int ctas, FUnit* out, int* off) {
  std::vector<std::pair<double, int>> cost(u.size());
  for (size_t i = 0; i < u.size(); ++i) {
    const HlrgInst& q = inst[act[u[i].inst]];
    cost[i] = {(double)(u[i].r1 - u[i].r0) * (2.0 + q.Dp / 64), (int)i};
  }
  std::stable_sort(cost.begin(), cost.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
    return a.first > b.first;
  });
  std::vector<double> load(ctas, 0.0);
  std::vector<std::vector<int>> lists(ctas);
  for (const auto& c : cost) {
    int best = 0;
    for (int j = 1; j < ctas; ++j)
      if (load[j] < load[best]) best = j;
    load[best] += c.first;
    lists[best].push_back(c.second);
  }
  int k = 0;
  for (int j = 0; j < ctas; ++j) {
    off[j] = k;
    for (int i : lists[j]) out[k++] = u[i];
  }
  off[ctas] = k;
}
}  // namespace
}  // namespace ab

extern "C" int ab_hlrg_create(int n, const ab_hlrb_model* models, const int* C, ab_hlrg** out) {
  using namespace ab;
  AB_REQUIRE(out && models && C, AB_ERR_ARG, "ab_hlrg_create: null argument");
  *out = nullptr;
  AB_REQUIRE(n >= 1 && n <= tc::GROUP_MAX, AB_ERR_ARG, "ab_hlrg_create: n must be 1..%d (got %d)", tc::GROUP_MAX, n);
  std::unique_ptr<ab_hlrg> g(new ab_hlrg());
  g->inst.resize(n);
  g->fused = true;
  for (int i = 0; i < n; ++i) {
    int rc = hlrb_check_model(&models[i]);
    if (rc) return rc;
    AB_REQUIRE(C[i] > 0 && C[i] <= 65535, AB_ERR_ARG, "ab_hlrg_create: instance %d: C must be 1..65535", i);
    AB_REQUIRE(models[i].D % 8 == 0, AB_ERR_ARG, "ab_hlrg_create: instance %d: D must be a multiple of 8", i);
    if (models[i].D > F_MAX_D) g->fused = false;
  }
  size_t wtot = 0;
  std::vector<size_t> woff(n);
  long long fwd_tiles = 0, bwd_tiles = 0;
  for (int i = 0; i < n; ++i) {
    HlrgInst& q = g->inst[i];
    q.m = models[i];
    q.C = C[i];
    q.L = layout(q.m.N, q.m.D, q.C, nullptr);
    AB_REQUIRE(q.L.fwd_bn == 256 && q.L.groups == 2 && q.L.bn <= G_BWD_BN, AB_ERR_STATE,
               "ab_hlrg_create: built-in launch shape changed");
    q.Dp = q.L.Dp;
    q.Dn = (q.m.D + 15) / 16 * 16;
    q.rtiles = (q.m.N + F_ROWS - 1) / F_ROWS;
    q.nseg = (q.rtiles + F_SEG_TILES - 1) / F_SEG_TILES;
    size_t o = 0;
    q.f_t3 = o;  o = al256(o + (size_t)q.C * 3 * q.Dp * 2);
    q.f_llp = o; o = al256(o + (size_t)q.nseg * F_GROUPS * q.C * 4);
    q.f_gw = o;  o = al256(o + (size_t)q.nseg * q.C * q.Dn * 4);
    q.f_total = o;
    woff[i] = wtot;
    wtot = al256(wtot + (g->fused ? q.f_total : q.L.total));
    g->C_max = std::max(g->C_max, q.C);
    g->Dp_max = std::max(g->Dp_max, q.L.Dp);
    g->units_max += ((q.C + tc::BM - 1) / tc::BM) * q.nseg;
  }
  AB_CUDA(cudaMalloc(&g->work, wtot));
  if (g->fused) g->finst.resize(n);
  for (int i = 0; i < n; ++i) {
    HlrgInst& q = g->inst[i];
    const Layout& L = q.L;
    q.work = g->work + woff[i];
    int rc;
    if (g->fused) {
      FInst& f = g->finst[i];
      std::memset(&f, 0, sizeof(f));
      __nv_bfloat16* t3 = reinterpret_cast<__nv_bfloat16*>(q.work + q.f_t3);
      const int nb = L.Np / 64;
      if ((rc = tc::encode_2d_bf16(&f.t3, t3, q.C, 3 * q.Dp, 3 * q.Dp, tc::BM))) return rc;
      if ((rc = tc::encode_2d_bf16(&f.x, q.m.X, q.m.N, q.m.D, q.m.ldx, F_ROWS))) return rc;
      if ((rc = tc::encode_2d_bf16(&f.xt, q.m.Xt, (uint64_t)nb * q.m.D, 64, 64, q.Dn))) return rc;
      f.y = q.m.y;
      f.llp = reinterpret_cast<float*>(q.work + q.f_llp);
      f.gw = reinterpret_cast<float*>(q.work + q.f_gw);
      f.N = q.m.N;
      f.D = q.m.D;
      f.Dp = q.Dp;
      f.Dn = q.Dn;
      f.C = q.C;
      continue;
    }
    __nv_bfloat16* t3 = reinterpret_cast<__nv_bfloat16*>(q.work + L.off_t3);
    __nv_bfloat16* r3 = reinterpret_cast<__nv_bfloat16*>(q.work + L.off_r3);
    float* llp = reinterpret_cast<float*>(q.work + L.off_ll);
    float* w = reinterpret_cast<float*>(q.work + L.off_w);
    if ((rc = tc::encode_2d_bf16(&q.fwd.ta, t3, q.C, 3 * L.Dp, 3 * L.Dp, tc::BM))) return rc;
    if ((rc = tc::encode_2d_bf16(&q.fwd.tb, q.m.X, q.m.N, q.m.D, q.m.ldx, L.fwd_bn))) return rc;
    q.fwd.sh = tc::make_shape(q.C, q.m.N, q.m.D, 1, tc::row_major(L.Dp), tc::row_major(0), L.fwd_bn);
    q.fwd.bn = L.fwd_bn;
    const int nb = L.Np / 64;
    if ((rc = tc::encode_2d_bf16(&q.bwd.ta, r3, (uint64_t)nb * R_PARTS * q.C, 64, 64, tc::BM))) return rc;
    if ((rc = tc::encode_2d_bf16(&q.bwd.tb, q.m.Xt, (uint64_t)nb * q.m.D, 64, 64, L.bn))) return rc;
    q.bwd.sh = tc::make_shape(q.C, q.m.D, q.m.N, L.splits, tc::k_blocked(R_PARTS, q.C), tc::k_blocked(1, q.m.D), L.bn);
    AB_REQUIRE(q.bwd.sh.splits == L.splits, AB_ERR_STATE, "ab_hlrg_create: split arithmetic mismatch");
    q.bwd.bn = L.bn;
    q.fe = GFwd{q.m.y, r3, llp, q.m.N, L.Np, q.C, nullptr, 0, 0.0f, 0.0f};
    q.ge = GradEpi{w, q.C, q.m.D, L.ldw, 0};
    fwd_tiles += (long long)q.fwd.sh.m_tiles * q.fwd.sh.n_tiles * q.fwd.sh.splits;
    bwd_tiles += (long long)q.bwd.sh.m_tiles * q.bwd.sh.n_tiles * q.bwd.sh.splits;
  }
  AB_REQUIRE(fwd_tiles < (1LL << 31) && bwd_tiles < (1LL << 31), AB_ERR_ARG, "ab_hlrg_create: too many tiles");
  g->grid_fwd = (int)std::max<long long>(1, std::min<long long>(fwd_tiles, tc::sm_count()));
  g->grid_bwd = (int)std::max<long long>(1, std::min<long long>(bwd_tiles, tc::sm_count()));
  g->grid_f = tc::sm_count();
  size_t o = al256(sizeof(GHeads));
  g->o_fwd = o; o = al256(o + sizeof(tc::GProblem) * n);
  g->o_bwd = o; o = al256(o + sizeof(tc::GProblem) * n);
  g->o_fe = o;  o = al256(o + sizeof(GFwd) * n);
  g->o_ge = o;  o = al256(o + sizeof(GradEpi) * n);
  g->o_sp = o;  o = al256(o + sizeof(GSplit) * n);
  g->o_fin = o; o = al256(o + sizeof(GFinish) * n);
  g->o_fi = o;  o = al256(o + sizeof(FInst) * n);
  g->o_fu = o;  o = al256(o + sizeof(FUnit) * (size_t)g->units_max);
  g->o_off = o; o = al256(o + sizeof(int) * (size_t)(g->grid_f + 1));
  g->bytes = o;
  AB_CUDA(cudaMalloc(&g->tab, g->bytes));
  AB_CUDA(cudaMemset(g->tab, 0, g->bytes));
  g->stage = static_cast<unsigned char*>(std::aligned_alloc(256, g->bytes));
  AB_REQUIRE(g->stage, AB_ERR_CUDA, "ab_hlrg_create: host allocation failed");
  std::memset(g->stage, 0, g->bytes);
  if (g->fused) {
    AB_CUDA(cudaFuncSetAttribute(hlrf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, F_SMEM));
  } else {
    using GF = tc::GCfg<256, 3, 1, GFwd>::C;
    using GB = tc::GCfg<G_BWD_BN, R_PARTS, 1, GradEpi>::C;
    static_assert(GF::SMEM_BYTES <= tc::SMEM_BUDGET && GB::SMEM_BYTES <= tc::SMEM_BUDGET,
                  "grouped tiles exceed shared memory");
    AB_CUDA(cudaFuncSetAttribute(tc::grouped_gemm_kernel<256, 3, 1, GFwd>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, GF::SMEM_BYTES));
    AB_CUDA(cudaFuncSetAttribute(tc::grouped_gemm_kernel<G_BWD_BN, R_PARTS, 1, GradEpi>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, GB::SMEM_BYTES));
  }
  *out = g.release();
  return AB_OK;
}

extern "C" int ab_hlrg_bind(ab_hlrg* g, int i, const float* theta, int ldt, double* logp, float* grad, int ldg) {
  AB_REQUIRE(g, AB_ERR_ARG, "ab_hlrg_bind: null group");
  AB_REQUIRE(i >= 0 && i < (int)g->inst.size(), AB_ERR_ARG, "ab_hlrg_bind: no instance %d", i);
  ab::HlrgInst& q = g->inst[i];
  AB_REQUIRE(theta && logp && grad, AB_ERR_ARG, "ab_hlrg_bind: null pointer");
  AB_REQUIRE(ldt >= q.m.D && ldg >= q.m.D, AB_ERR_ARG, "ab_hlrg_bind: leading dimension too small");
  q.theta = theta;
  q.ldt = ldt;
  q.logp = logp;
  q.grad = grad;
  q.ldg = ldg;
  g->ready = false;   // takes effect at the next ab_hlrg_set_active
  return AB_OK;
}

extern "C" int ab_hlrg_set_active(ab_hlrg* g, const int* active, void* stream) {
  using namespace ab;
  AB_REQUIRE(g && active, AB_ERR_ARG, "ab_hlrg_set_active: null argument");
  const int n = (int)g->inst.size();
  unsigned char* h = g->stage;
  tc::GProblem* fwd = reinterpret_cast<tc::GProblem*>(h + g->o_fwd);
  tc::GProblem* bwd = reinterpret_cast<tc::GProblem*>(h + g->o_bwd);
  GFwd* fe = reinterpret_cast<GFwd*>(h + g->o_fe);
  GradEpi* ge = reinterpret_cast<GradEpi*>(h + g->o_ge);
  GSplit* sp = reinterpret_cast<GSplit*>(h + g->o_sp);
  GFinish* fin = reinterpret_cast<GFinish*>(h + g->o_fin);
  FInst* fi = reinterpret_cast<FInst*>(h + g->o_fi);
  int k = 0, tf = 0, tb = 0;
  std::vector<int> act;
  std::vector<FUnit> units;
  for (int i = 0; i < n; ++i) {
    if (!active[i]) continue;
    const HlrgInst& q = g->inst[i];
    AB_REQUIRE(q.theta, AB_ERR_STATE, "ab_hlrg_set_active: instance %d is active but not bound", i);
    if (g->fused) {
      fi[k] = g->finst[i];
      fused_units(q, k, units);
      sp[k] = GSplit{q.theta, reinterpret_cast<__nv_bfloat16*>(q.work + q.f_t3), q.ldt, q.C, q.m.D, q.Dp};
      fin[k] = GFinish{reinterpret_cast<const float*>(q.work + q.f_llp), reinterpret_cast<const float*>(q.work + q.f_gw),
                       q.theta, q.logp, q.grad, q.m.prior_a, q.m.prior_b, q.C, q.m.D, F_GROUPS * q.nseg, q.nseg, q.Dn, q.ldt,
                       q.m.prior, q.ldg};
    } else {
      fwd[k] = q.fwd;
      fwd[k].tile0 = tf;
      tf += q.fwd.sh.m_tiles * q.fwd.sh.n_tiles * q.fwd.sh.splits;
      bwd[k] = q.bwd;
      bwd[k].tile0 = tb;
      tb += q.bwd.sh.m_tiles * q.bwd.sh.n_tiles * q.bwd.sh.splits;
      fe[k] = q.fe;
      ge[k] = q.ge;
      sp[k] = GSplit{q.theta, reinterpret_cast<__nv_bfloat16*>(q.work + q.L.off_t3), q.ldt, q.C, q.m.D, q.L.Dp};
      fin[k] = GFinish{reinterpret_cast<const float*>(q.work + q.L.off_ll),
                       reinterpret_cast<const float*>(q.work + q.L.off_w), q.theta, q.logp, q.grad, q.m.prior_a,
                       q.m.prior_b, q.C, q.m.D, q.L.fwd_tiles * q.L.groups, q.L.splits, q.L.ldw, q.ldt, q.m.prior,
                       q.ldg};
    }
    act.push_back(i);
    ++k;
  }
  if (g->fused)
    assign_units(units, g->inst, act, g->grid_f, reinterpret_cast<FUnit*>(h + g->o_fu),
                 reinterpret_cast<int*>(h + g->o_off));
  GHeads* hd = reinterpret_cast<GHeads*>(h);
  hd->fwd = tc::GHead{k, tf};
  hd->bwd = tc::GHead{k, tb};
  g->n_active = k;
  AB_CUDA(cudaMemcpyAsync(g->tab, h, g->bytes, cudaMemcpyHostToDevice, as_stream(stream)));
  g->ready = true;
  return AB_OK;
}

extern "C" int ab_hlrg_logp_grad(ab_hlrg* g, int* err, void* stream) {
  using namespace ab;
  AB_REQUIRE(g, AB_ERR_ARG, "ab_hlrg_logp_grad: null group");
  AB_REQUIRE(g->ready, AB_ERR_STATE, "ab_hlrg_logp_grad: call ab_hlrg_set_active after creating or binding");
  cudaStream_t st = as_stream(stream);
  const int n = (int)g->inst.size();
  const GHeads* head = reinterpret_cast<const GHeads*>(g->tab);
  hlrg_split_kernel<<<dim3(ceil_div(g->Dp_max, 256), g->C_max, n), 256, 0, st>>>(
      reinterpret_cast<const GSplit*>(g->tab + g->o_sp), head);
  AB_LAUNCH_CHECK("hlrg_split_kernel");
  if (g->fused) {
    hlrf_kernel<<<g->grid_f, F_THREADS, F_SMEM, st>>>(reinterpret_cast<const FInst*>(g->tab + g->o_fi),
                                                      reinterpret_cast<const FUnit*>(g->tab + g->o_fu),
                                                      reinterpret_cast<const int*>(g->tab + g->o_off), err);
    AB_LAUNCH_CHECK("hlrf_kernel");
  } else {
    using GF = tc::GCfg<256, 3, 1, GFwd>::C;
    using GB = tc::GCfg<G_BWD_BN, R_PARTS, 1, GradEpi>::C;
    tc::grouped_gemm_kernel<256, 3, 1, GFwd><<<g->grid_fwd, tc::threads_for(GFwd::kWarps), GF::SMEM_BYTES, st>>>(
        reinterpret_cast<const tc::GProblem*>(g->tab + g->o_fwd), reinterpret_cast<const GFwd*>(g->tab + g->o_fe),
        &head->fwd, err);
    AB_LAUNCH_CHECK("grouped_gemm_kernel (forward)");
    tc::grouped_gemm_kernel<G_BWD_BN, R_PARTS, 1, GradEpi>
        <<<g->grid_bwd, tc::threads_for(GradEpi::kWarps), GB::SMEM_BYTES, st>>>(
            reinterpret_cast<const tc::GProblem*>(g->tab + g->o_bwd),
            reinterpret_cast<const GradEpi*>(g->tab + g->o_ge), &head->bwd, err);
    AB_LAUNCH_CHECK("grouped_gemm_kernel (backward)");
  }
  hlrg_finish_kernel<<<dim3(g->C_max, n), 256, 0, st>>>(reinterpret_cast<const GFinish*>(g->tab + g->o_fin), head);
  AB_LAUNCH_CHECK("hlrg_finish_kernel");
  return AB_OK;
}

extern "C" int ab_hlrg_fused(const ab_hlrg* g) { return g && g->fused ? 1 : 0; }

extern "C" int ab_hlrg_destroy(ab_hlrg* g) {
  delete g;
  return AB_OK;
}
