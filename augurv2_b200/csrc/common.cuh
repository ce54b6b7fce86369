// Shared helpers of the CUDA library: status codes, the per-thread error
// string behind ab_last_error(), launch checking and warp utilities.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>

#include "../../include/augur_b200.h"

namespace ab {

// Records a formatted message as the calling thread's last error and returns
// the status code, so call sites read `return fail(AB_ERR_ARG, "...")`.
int fail(int code, const char* fmt, ...);

// Converts a CUDA error into a status, recording where it came from.
int cuda_status(cudaError_t e, const char* what);

#define AB_CUDA(call)                                           \
  do {                                                          \
    cudaError_t _e = (call);                                    \
    if (_e != cudaSuccess) return ::ab::cuda_status(_e, #call); \
  } while (0)

#define AB_LAUNCH_CHECK(name)                                   \
  do {                                                          \
    cudaError_t _e = cudaGetLastError();                        \
    if (_e != cudaSuccess) return ::ab::cuda_status(_e, name);  \
  } while (0)

#define AB_REQUIRE(cond, code, ...)                             \
  do {                                                          \
    if (!(cond)) return ::ab::fail((code), __VA_ARGS__);        \
  } while (0)

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum_f32(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order block sum: warp butterflies, then warp 0 adds the warp
// partials in warp order.  The result is deterministic for a given launch
// shape and is broadcast to every thread.  `red` holds >= 33 doubles.
__device__ __forceinline__ double block_sum_f64(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum_f64(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < nw ? red[lane] : 0.0;
    t = warp_sum_f64(t);
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

static inline unsigned int ceil_div(size_t a, size_t b) { return (unsigned int)((a + b - 1) / b); }

}  // namespace ab
