// Gradient surrogate network: a small MLP d_in -> h1 -> h2 -> d_out with
// exact (erf) GELU after the two hidden layers, trained online by the
// sampler on (position, gradient) pairs.  No counterpart in the reference,
// whose samplers always evaluate the exact gradient.
//
// Parameters are one flat FP32 master vector
//   [W1 (h1 x d_in), b1 (h1), W2 (h2 x h1), b2 (h2), W3 (d_out x h2), b3 (d_out)]
// with a bf16 copy of the same layout; forward passes multiply by the bf16
// weights with FP32 accumulation and FP32 biases.  The layer products run on
// the CUDA cores (64 x 64 output tiles, 16-deep K slices staged in shared
// memory, 4 x 4 outputs per thread): they are a few hundred MFLOP per step,
// small beside the exact HLR pass.
//
//   forward   P1 = X W1^T + b1, A1 = gelu(P1), P2 = A1 W2^T + b2,
//             A2 = gelu(P2), Y = A2 W3^T + b3 — one fused launch, a few rows
//             per block with the activations in shared memory
//   loss      mean squared error against a target, dY = 2 (Y - T) / (B d_out)
//   backward  dW3 = dY^T A2, db3 = colsum dY, dP2 = (dY W3) . gelu'(P2), ...
//   Adam      on the master vector, refreshing the bf16 copy.
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"

namespace ab {
namespace {

constexpr int TM = 64, TN = 64, TK = 16;

__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

enum { EPI_STORE = 0, EPI_GELU = 1, EPI_GELU_GRAD = 2 };

// C[m][n] = sum_k A(m, k) B(k, n) (+ bias[n]) with A(m, k) = A[m*sam + k*sak]
// and B(k, n) = B[k*sbk + n*sbn].  EPI_GELU also stores P (pre-activation)
// to C and gelu(P) to C2; EPI_GELU_GRAD multiplies by gelu'(P[m][n]).
template <typename TB, int EPI>
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const float* __restrict__ A, int sam,
                                                       int sak, const TB* __restrict__ B, int sbk, int sbn,
                                                       const float* __restrict__ bias, float* __restrict__ C,
                                                       int ldc, float* __restrict__ C2, const float* __restrict__ P,
                                                       int ldp) {
  __shared__ float As[TK][TM + 4];
  __shared__ float Bs[TK][TN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  // consecutive threads walk the operand's unit-stride dimension
  const bool a_k_unit = sak == 1, b_k_unit = sbk == 1;
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int e = threadIdx.x; e < TK * TM; e += 256) {
      const int kk = a_k_unit ? e % TK : e / TM, mm = a_k_unit ? e / TK : e % TM;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[(size_t)m * sam + (size_t)k * sak] : 0.0f;
    }
    for (int e = threadIdx.x; e < TK * TN; e += 256) {
      const int kk = b_k_unit ? e % TK : e / TN, nn = b_k_unit ? e / TK : e % TN;
      const int n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < N && k < K) ? ld(B + (size_t)k * sbk + (size_t)n * sbn) : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      float v = acc[i][j];
      if (EPI != EPI_GELU_GRAD && bias) v += bias[n];
      if (EPI == EPI_STORE) {
        C[(size_t)m * ldc + n] = v;
      } else if (EPI == EPI_GELU) {
        C[(size_t)m * ldc + n] = v;
        C2[(size_t)m * ldc + n] = gelu(v);
      } else {
        C[(size_t)m * ldc + n] = v * gelu_grad(P[(size_t)m * ldp + n]);
      }
    }
  }
}

// out[n] = sum_m X[m][n], sequential over m (deterministic).
__global__ void colsum_kernel(int M, int N, const float* __restrict__ X, int ldx, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int m = 0; m < M; ++m) s += X[(size_t)m * ldx + n];
  out[n] = s;
}

// dY = 2 (Y - T) / (B d), and the per-row squared error (FP64).
__global__ void mse_kernel(int B, int D, const float* __restrict__ Y, int ldy, const float* __restrict__ T, int ldt,
                           float* __restrict__ dY, double* __restrict__ row_sq) {
  __shared__ double red[33];
  const int b = blockIdx.x;
  const float scale = 2.0f / ((float)B * (float)D);
  double s = 0.0;
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    const float e = Y[(size_t)b * ldy + d] - T[(size_t)b * ldt + d];
    dY[(size_t)b * D + d] = scale * e;
    s += (double)e * (double)e;
  }
  s = block_sum_f64(s, red);
  if (threadIdx.x == 0) row_sq[b] = s;
}

__global__ void adam_kernel(size_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                            __nv_bfloat16* __restrict__ wb) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void to_bf16_kernel(size_t n, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    wb[i] = __float2bfloat16_rn(w[i]);
}

// z = (theta - mu) * inv_s, per coordinate.
__global__ void sur_pre_kernel(int C, int D, const float* __restrict__ theta, const float* __restrict__ mu,
                               const float* __restrict__ inv_s, float* __restrict__ z) {
  const size_t n = (size_t)C * D;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int d = (int)(i % D);
    z[i] = (theta[i] - mu[d]) * inv_s[d];
  }
}

// g = a + h * (theta - mu) + o * out: the diagonal linear part plus the
// network's correction in output units o.
__global__ void sur_post_kernel(int C, int D, const float* __restrict__ theta, const float* __restrict__ out,
                                const float* __restrict__ mu, const float* __restrict__ a,
                                const float* __restrict__ h, const float* __restrict__ o, float* __restrict__ g) {
  const size_t n = (size_t)C * D;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int d = (int)(i % D);
    g[i] = a[d] + h[d] * (theta[i] - mu[d]) + o[d] * out[i];
  }
}

// One dense layer for G rows held in shared memory: out[g][j] = act(b[j] +
// sum_k W[j][k] in[g][k]).  One output feature j per thread: the thread
// walks its bf16 weight row in 16-byte pieces (consecutive pieces share a
// cache line) and reads the G input rows as shared-memory broadcasts, so no
// cross-lane reduction is needed and the sum order is fixed.
template <int G>
__device__ __forceinline__ void dense_layer(const float* __restrict__ in, int din, const __nv_bfloat16* __restrict__ W,
                                            const float* __restrict__ b, int dout, float* __restrict__ out,
                                            float* __restrict__ pre, bool gelu_act) {
  for (int j = threadIdx.x; j < dout; j += blockDim.x) {
    float acc[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = 0.0f;
    const uint4* row = reinterpret_cast<const uint4*>(W + (size_t)j * din);
    const int n8 = din >> 3;
#pragma unroll 4
    for (int k8 = 0; k8 < n8; ++k8) {
      const uint4 raw = __ldg(row + k8);
      const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&raw);
      float wv[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 f = __bfloat1622float2(h2[i]);
        wv[2 * i] = f.x;
        wv[2 * i + 1] = f.y;
      }
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const float4 x0 = *reinterpret_cast<const float4*>(in + g * din + 8 * k8);
        const float4 x1 = *reinterpret_cast<const float4*>(in + g * din + 8 * k8 + 4);
        acc[g] = fmaf(wv[0], x0.x, acc[g]);
        acc[g] = fmaf(wv[1], x0.y, acc[g]);
        acc[g] = fmaf(wv[2], x0.z, acc[g]);
        acc[g] = fmaf(wv[3], x0.w, acc[g]);
        acc[g] = fmaf(wv[4], x1.x, acc[g]);
        acc[g] = fmaf(wv[5], x1.y, acc[g]);
        acc[g] = fmaf(wv[6], x1.z, acc[g]);
        acc[g] = fmaf(wv[7], x1.w, acc[g]);
      }
    }
    const float bj = b[j];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const float v = acc[g] + bj;
      if (pre) pre[g * dout + j] = v;
      out[g * dout + j] = gelu_act ? gelu(v) : v;
    }
  }
}

// The whole network for G rows per block.  SUR: input theta with the
// surrogate's input map z = (theta - mu) * inv_s, output the gradient
// estimate a + h (theta - mu) + o * y; otherwise input x, output y, and the
// activations (P1, A1, P2, A2 by rows) saved for the backward pass when act
// is not NULL.
template <int G, bool SUR>
__global__ void __launch_bounds__(256) mlp_fused_kernel(int B, int din, int h1, int h2, int dout,
                                                        const float* __restrict__ x, int ldx,
                                                        const __nv_bfloat16* __restrict__ wb,
                                                        const float* __restrict__ w, float* __restrict__ y, int ldy,
                                                        float* __restrict__ act, const float* __restrict__ mu,
                                                        const float* __restrict__ inv_s, const float* __restrict__ sa,
                                                        const float* __restrict__ sh, const float* __restrict__ so) {
  extern __shared__ float sm[];
  float* z = sm;                       // [G][din]
  float* a1 = z + G * din;             // [G][h1]
  float* a2 = a1 + G * h1;             // [G][h2]
  float* p1 = a2 + G * h2;             // [G][h1]
  float* p2 = p1 + G * h1;             // [G][h2]
  float* o3 = p2 + G * h2;             // [G][dout]
  const int r0 = blockIdx.x * G;
  const size_t ow1 = 0, ob1 = (size_t)h1 * din, ow2 = ob1 + h1, ob2 = ow2 + (size_t)h2 * h1, ow3 = ob2 + h2,
               ob3 = ow3 + (size_t)dout * h2;
  for (int i = threadIdx.x; i < G * din; i += blockDim.x) {
    const int g = i / din, k = i % din, r = r0 + g;
    float v = 0.0f;
    if (r < B) {
      v = x[(size_t)r * ldx + k];
      if (SUR) v = (v - mu[k]) * inv_s[k];
    }
    z[i] = v;
  }
  __syncthreads();
  const bool save = !SUR && act;
  dense_layer<G>(z, din, wb + ow1, w + ob1, h1, a1, save ? p1 : nullptr, true);
  __syncthreads();
  dense_layer<G>(a1, h1, wb + ow2, w + ob2, h2, a2, save ? p2 : nullptr, true);
  __syncthreads();
  dense_layer<G>(a2, h2, wb + ow3, w + ob3, dout, o3, nullptr, false);
  __syncthreads();
  for (int i = threadIdx.x; i < G * dout; i += blockDim.x) {
    const int g = i / dout, j = i % dout, r = r0 + g;
    if (r >= B) continue;
    float v = o3[i];
    if (SUR) {
      const float th = x[(size_t)r * ldx + j];
      v = sa[j] + sh[j] * (th - mu[j]) + so[j] * v;
    }
    y[(size_t)r * ldy + j] = v;
  }
  if (save) {
    float* P1 = act;
    float* A1 = P1 + (size_t)B * h1;
    float* P2 = A1 + (size_t)B * h1;
    float* A2 = P2 + (size_t)B * h2;
    for (int i = threadIdx.x; i < G * h1; i += blockDim.x) {
      const int g = i / h1, j = i % h1, r = r0 + g;
      if (r < B) {
        P1[(size_t)r * h1 + j] = p1[i];
        A1[(size_t)r * h1 + j] = a1[i];
      }
    }
    for (int i = threadIdx.x; i < G * h2; i += blockDim.x) {
      const int g = i / h2, j = i % h2, r = r0 + g;
      if (r < B) {
        P2[(size_t)r * h2 + j] = p2[i];
        A2[(size_t)r * h2 + j] = a2[i];
      }
    }
  }
}

constexpr int FUSED_G = 4;

template <bool SUR>
int launch_fused(const ab_mlp_desc* d, int B, const float* x, int ldx, float* y, int ldy, float* act,
                 const float* mu, const float* inv_s, const float* a, const float* h, const float* o,
                 cudaStream_t st) {
  const size_t smem = sizeof(float) * FUSED_G * ((size_t)d->d_in + 2 * d->h1 + 2 * d->h2 + d->d_out);
  AB_REQUIRE(smem <= 200 * 1024, AB_ERR_ARG, "mlp: layers too wide for the fused kernel");
  AB_CUDA(cudaFuncSetAttribute(mlp_fused_kernel<FUSED_G, SUR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  mlp_fused_kernel<FUSED_G, SUR><<<ceil_div(B, FUSED_G), 256, smem, st>>>(
      B, d->d_in, d->h1, d->h2, d->d_out, x, ldx, static_cast<const __nv_bfloat16*>(d->wb), d->w, y, ldy, act, mu,
      inv_s, a, h, o);
  AB_LAUNCH_CHECK("mlp_fused_kernel");
  return AB_OK;
}

struct Offsets {
  size_t w1, b1, w2, b2, w3, b3, total;
};

Offsets offsets(const ab_mlp_desc* d) {
  Offsets o;
  size_t k = 0;
  o.w1 = k; k += (size_t)d->h1 * d->d_in;
  o.b1 = k; k += d->h1;
  o.w2 = k; k += (size_t)d->h2 * d->h1;
  o.b2 = k; k += d->h2;
  o.w3 = k; k += (size_t)d->d_out * d->h2;
  o.b3 = k; k += d->d_out;
  o.total = k;
  return o;
}

template <typename TB, int EPI>
int gemm(int M, int N, int K, const float* A, int sam, int sak, const TB* B, int sbk, int sbn, const float* bias,
         float* C, int ldc, float* C2, const float* P, int ldp, cudaStream_t st) {
  dim3 grid(ceil_div(N, TN), ceil_div(M, TM));
  mlp_gemm_kernel<TB, EPI><<<grid, 256, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, ldc, C2, P, ldp);
  AB_LAUNCH_CHECK("mlp_gemm_kernel");
  return AB_OK;
}

int check(const ab_mlp_desc* d) {
  AB_REQUIRE(d, AB_ERR_ARG, "mlp: null descriptor");
  AB_REQUIRE(d->d_in > 0 && d->h1 > 0 && d->h2 > 0 && d->d_out > 0, AB_ERR_ARG, "mlp: bad layer sizes");
  AB_REQUIRE(d->d_in % 8 == 0 && d->h1 % 8 == 0 && d->h2 % 8 == 0 && d->d_out % 8 == 0, AB_ERR_ARG,
             "mlp: layer widths must be multiples of 8");
  AB_REQUIRE((reinterpret_cast<uintptr_t>(d->wb) & 15) == 0, AB_ERR_ARG, "mlp: bf16 weights must be 16-byte aligned");
  AB_REQUIRE(d->w && d->wb, AB_ERR_ARG, "mlp: null parameters");
  return AB_OK;
}

}  // namespace
}  // namespace ab

using namespace ab;

extern "C" size_t ab_mlp_param_count(int d_in, int h1, int h2, int d_out) {
  if (d_in <= 0 || h1 <= 0 || h2 <= 0 || d_out <= 0) return 0;
  return (size_t)h1 * d_in + h1 + (size_t)h2 * h1 + h2 + (size_t)d_out * h2 + d_out;
}

extern "C" size_t ab_mlp_act_floats(int B, int h1, int h2) {
  if (B <= 0 || h1 <= 0 || h2 <= 0) return 0;
  return (size_t)B * (2 * (size_t)h1 + 2 * (size_t)h2);
}

extern "C" int ab_mlp_forward(const ab_mlp_desc* d, int B, const float* x, int ldx, float* y, int ldy, float* act,
                              void* stream) {
  int rc = check(d);
  if (rc) return rc;
  AB_REQUIRE(B > 0 && x && y && ldx >= d->d_in && ldy >= d->d_out && ldx % 4 == 0, AB_ERR_ARG,
             "ab_mlp_forward: bad arguments");
  return launch_fused<false>(d, B, x, ldx, y, ldy, act, nullptr, nullptr, nullptr, nullptr, nullptr,
                             as_stream(stream));
}

extern "C" int ab_sur_predict(const ab_mlp_desc* d, int C, const float* theta, int ldt, const float* mu,
                              const float* inv_s, const float* a, const float* h, const float* o, float* g, int ldg,
                              void* stream) {
  int rc = check(d);
  if (rc) return rc;
  AB_REQUIRE(d->d_in == d->d_out, AB_ERR_ARG, "ab_sur_predict: the network must map D to D");
  AB_REQUIRE(C > 0 && theta && mu && inv_s && a && h && o && g && ldt >= d->d_in && ldg >= d->d_out, AB_ERR_ARG,
             "ab_sur_predict: bad arguments");
  return launch_fused<true>(d, C, theta, ldt, g, ldg, nullptr, mu, inv_s, a, h, o, as_stream(stream));
}

extern "C" int ab_mlp_mse(int B, int D, const float* y, int ldy, const float* target, int ldt, float* dy,
                          double* row_sq, void* stream) {
  AB_REQUIRE(B > 0 && D > 0 && y && target && dy && row_sq && ldy >= D && ldt >= D, AB_ERR_ARG,
             "ab_mlp_mse: bad arguments");
  mse_kernel<<<B, 256, 0, as_stream(stream)>>>(B, D, y, ldy, target, ldt, dy, row_sq);
  AB_LAUNCH_CHECK("mse_kernel");
  return AB_OK;
}

extern "C" size_t ab_mlp_backward_scratch_floats(int B, int h1, int h2) {
  if (B <= 0 || h1 <= 0 || h2 <= 0) return 0;
  return (size_t)B * ((size_t)h1 + (size_t)h2);
}

extern "C" int ab_mlp_backward(const ab_mlp_desc* d, int B, const float* x, int ldx, const float* dy,
                               const float* act, float* grad, float* scratch, void* stream) {
  int rc = check(d);
  if (rc) return rc;
  AB_REQUIRE(B > 0 && x && dy && act && grad && scratch && ldx >= d->d_in, AB_ERR_ARG,
             "ab_mlp_backward: bad arguments");
  const Offsets o = offsets(d);
  const __nv_bfloat16* wb = static_cast<const __nv_bfloat16*>(d->wb);
  cudaStream_t st = as_stream(stream);
  const float* P1 = act;
  const float* A1 = P1 + (size_t)B * d->h1;
  const float* P2 = A1 + (size_t)B * d->h1;
  const float* A2 = P2 + (size_t)B * d->h2;
  float* dP2 = scratch;                        // [B][h2]
  float* dP1 = scratch + (size_t)B * d->h2;    // [B][h1]
  const int h1 = d->h1, h2 = d->h2, din = d->d_in, dout = d->d_out;
  // dW3[o][j] = sum_b dY[b][o] A2[b][j];  db3 = colsum dY
  if ((rc = gemm<float, EPI_STORE>(dout, h2, B, dy, 1, dout, A2, h2, 1, nullptr, grad + o.w3, h2, nullptr, nullptr, 0,
                                   st)))
    return rc;
  colsum_kernel<<<ceil_div(dout, 128), 128, 0, st>>>(B, dout, dy, dout, grad + o.b3);
  AB_LAUNCH_CHECK("colsum_kernel");
  // dP2 = (dY W3) . gelu'(P2)
  if ((rc = gemm<__nv_bfloat16, EPI_GELU_GRAD>(B, h2, dout, dy, dout, 1, wb + o.w3, h2, 1, nullptr, dP2, h2, nullptr,
                                               P2, h2, st)))
    return rc;
  if ((rc = gemm<float, EPI_STORE>(h2, h1, B, dP2, 1, h2, A1, h1, 1, nullptr, grad + o.w2, h1, nullptr, nullptr, 0,
                                   st)))
    return rc;
  colsum_kernel<<<ceil_div(h2, 128), 128, 0, st>>>(B, h2, dP2, h2, grad + o.b2);
  AB_LAUNCH_CHECK("colsum_kernel");
  // dP1 = (dP2 W2) . gelu'(P1)
  if ((rc = gemm<__nv_bfloat16, EPI_GELU_GRAD>(B, h1, h2, dP2, h2, 1, wb + o.w2, h1, 1, nullptr, dP1, h1, nullptr, P1,
                                               h1, st)))
    return rc;
  if ((rc = gemm<float, EPI_STORE>(h1, din, B, dP1, 1, h1, x, ldx, 1, nullptr, grad + o.w1, din, nullptr, nullptr, 0,
                                   st)))
    return rc;
  colsum_kernel<<<ceil_div(h1, 128), 128, 0, st>>>(B, h1, dP1, h1, grad + o.b1);
  AB_LAUNCH_CHECK("colsum_kernel");
  return AB_OK;
}

extern "C" int ab_mlp_adam(const ab_mlp_desc* d, const float* grad, float* m, float* v, int step, float lr, float b1,
                           float b2, float eps, void* stream) {
  int rc = check(d);
  if (rc) return rc;
  AB_REQUIRE(grad && m && v && step >= 1 && lr > 0.0f, AB_ERR_ARG, "ab_mlp_adam: bad arguments");
  const size_t n = ab_mlp_param_count(d->d_in, d->h1, d->h2, d->d_out);
  const float c1 = (float)(1.0 / (1.0 - pow((double)b1, step)));
  const float c2 = (float)(1.0 / (1.0 - pow((double)b2, step)));
  adam_kernel<<<ceil_div(n, 256 * 4), 256, 0, as_stream(stream)>>>(n, d->w, grad, m, v, lr, b1, b2, eps, c1, c2,
                                                                    static_cast<__nv_bfloat16*>(d->wb));
  AB_LAUNCH_CHECK("adam_kernel");
  return AB_OK;
}

extern "C" int ab_mlp_sync_bf16(const ab_mlp_desc* d, void* stream) {
  int rc = check(d);
  if (rc) return rc;
  const size_t n = ab_mlp_param_count(d->d_in, d->h1, d->h2, d->d_out);
  to_bf16_kernel<<<ceil_div(n, 256 * 4), 256, 0, as_stream(stream)>>>(n, d->w, static_cast<__nv_bfloat16*>(d->wb));
  AB_LAUNCH_CHECK("to_bf16_kernel");
  return AB_OK;
}

extern "C" int ab_sur_pre(int C, int D, const float* theta, const float* mu, const float* inv_s, float* z,
                          void* stream) {
  AB_REQUIRE(C > 0 && D > 0 && theta && mu && inv_s && z, AB_ERR_ARG, "ab_sur_pre: bad arguments");
  sur_pre_kernel<<<ceil_div((size_t)C * D, 1024), 256, 0, as_stream(stream)>>>(C, D, theta, mu, inv_s, z);
  AB_LAUNCH_CHECK("sur_pre_kernel");
  return AB_OK;
}

extern "C" int ab_sur_post(int C, int D, const float* theta, const float* out, const float* mu, const float* a,
                           const float* h, const float* o, float* g, void* stream) {
  AB_REQUIRE(C > 0 && D > 0 && theta && out && mu && a && h && o && g, AB_ERR_ARG, "ab_sur_post: bad arguments");
  sur_post_kernel<<<ceil_div((size_t)C * D, 1024), 256, 0, as_stream(stream)>>>(C, D, theta, out, mu, a, h, o, g);
  AB_LAUNCH_CHECK("sur_post_kernel");
  return AB_OK;
}
