// Host side of the tensor-core GEMM core: tensor maps, launch helpers, and a
// plain "store" epilogue exposed through the C ABI for checking the core
// against a reference matrix product.
#include <cudaTypedefs.h>
#include <mutex>

#include "common.cuh"
#include "tc_gemm.cuh"
#include "tc_host.cuh"

namespace ab {
namespace tc {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mu;
int g_sms[64] = {0};
}  // namespace

int sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!g_sms[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    g_sms[dev] = n;
  }
  return g_sms[dev];
}

int encode_2d_bf16(CUtensorMap* map, const void* ptr, uint64_t rows, uint64_t cols, uint64_t ld_elems,
                   uint32_t box_rows) {
  {
    std::lock_guard<std::mutex> lk(g_encode_mu);
    if (!g_encode) {
      cudaDriverEntryPointQueryResult q;
      void* fn = nullptr;
      AB_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q));
      AB_REQUIRE(fn && q == cudaDriverEntryPointSuccess, AB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
  }
  AB_REQUIRE((reinterpret_cast<uintptr_t>(ptr) & 15) == 0, AB_ERR_ARG, "tensor base must be 16-byte aligned");
  AB_REQUIRE((ld_elems * 2) % 16 == 0, AB_ERR_ARG, "row stride must be a multiple of 16 bytes");
  AB_REQUIRE(box_rows >= 1 && box_rows <= 256, AB_ERR_ARG, "box rows must be 1..256");
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {ld_elems * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  AB_REQUIRE(r == CUDA_SUCCESS, AB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return AB_OK;
}

// C (fp32, ldc) = A B^T, optionally split-K with atomic accumulation.
struct StoreEpi {
  static constexpr int kSmem = 0;
  static constexpr int kWarps = 4;
  float* C;
  int M, N, ldc;
  int atomic;
  __device__ void begin(int, int, int, char*, int) {}
  __device__ void rows(int row, int col0, const float* v, bool ok) {
    if (!ok) return;
    float* out = C + (size_t)row * ldc;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int c = col0 + i;
      if (c < N) {
        if (atomic) atomicAdd(out + c, v[i]);
        else out[c] = v[i];
      }
    }
  }
  __device__ void end(int, int, int, int, bool, int) {}
};

// Self-test of the bounded wait: one thread waits on an mbarrier that
// expects an arrival nothing makes, through the same routine the GEMM
// pipeline uses, and records AB_ERR_TIMEOUT and the cycles it waited.
__global__ void wait_probe_kernel(long long limit, int* status, long long* cycles) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  const long long t0 = clock64();
  const bool ok = mbar_wait_for(&bar, 0, limit);
  *cycles = clock64() - t0;
  *status = ok ? AB_OK : AB_ERR_TIMEOUT;
}

}  // namespace tc
}  // namespace ab

using namespace ab;
using namespace ab::tc;

extern "C" int ab_tc_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C,
                               int ldc, int splits, int* err, void* stream) {
  AB_REQUIRE(M > 0 && N > 0 && K > 0 && splits >= 1, AB_ERR_ARG, "ab_tc_gemm_bf16: bad sizes");
  AB_REQUIRE(A && B && C, AB_ERR_ARG, "ab_tc_gemm_bf16: null pointer");
  AB_REQUIRE(lda >= K && ldb >= K && ldc >= N, AB_ERR_ARG, "ab_tc_gemm_bf16: leading dimension too small");
  CUtensorMap ta, tb;
  int rc = encode_2d_bf16(&ta, A, M, K, lda, BM);
  if (rc) return rc;
  const int BN = N >= 256 ? 256 : (N > 64 ? 128 : 64);
  rc = encode_2d_bf16(&tb, B, N, K, ldb, BN);
  if (rc) return rc;
  const Shape sh = make_shape(M, N, K, splits, row_major(0), row_major(0), BN);
  StoreEpi epi{C, M, N, ldc, sh.splits > 1};
  cudaStream_t st = as_stream(stream);
  if (sh.splits > 1) AB_CUDA(cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * ldc, st));
  if (BN == 256) rc = launch_gemm<256, 1, 1>(ta, tb, sh, epi, err, st);
  else if (BN == 128) rc = launch_gemm<128, 1, 1>(ta, tb, sh, epi, err, st);
  else rc = launch_gemm<64, 1, 1>(ta, tb, sh, epi, err, st);
  return rc;
}

extern "C" int ab_tc_wait_probe(long long limit_cycles, int* status, long long* cycles, void* stream) {
  AB_REQUIRE(limit_cycles > 0 && limit_cycles <= ab::tc::WAIT_CYCLES, AB_ERR_ARG,
             "ab_tc_wait_probe: limit must be in (0, %lld] cycles", (long long)ab::tc::WAIT_CYCLES);
  AB_REQUIRE(status && cycles, AB_ERR_ARG, "ab_tc_wait_probe: null output");
  ab::tc::wait_probe_kernel<<<1, 32, 0, ab::as_stream(stream)>>>(limit_cycles, status, cycles);
  AB_LAUNCH_CHECK("wait_probe_kernel");
  return AB_OK;
}
