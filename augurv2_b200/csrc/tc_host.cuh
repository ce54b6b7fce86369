// Host helpers of the tensor-core GEMM core (tensor maps, launches).
#pragma once
#include "common.cuh"
#include "tc_gemm.cuh"

namespace ab {
namespace tc {

// Row-major bf16 matrix [rows][ld] -> tensor map with 64-column x box_rows
// boxes, 128-byte swizzle (the layout make_desc describes).
int encode_2d_bf16(CUtensorMap* map, const void* ptr, uint64_t rows, uint64_t cols, uint64_t ld_elems,
                   uint32_t box_rows);

template <int BN, class Epi>
int launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, int K, int ksplit, const Epi& epi,
                int* err, dim3 grid, cudaStream_t st) {
  using C = Cfg<BN>;
  const int smem = C::SMEM_BYTES + Epi::kSmem;
  AB_REQUIRE(smem <= 232448, AB_ERR_ARG, "GEMM tile needs %d bytes of shared memory", smem);
  AB_CUDA(cudaFuncSetAttribute(gemm_kernel<BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  gemm_kernel<BN, Epi><<<grid, 128, smem, st>>>(ta, tb, M, N, K, ksplit, epi, err);
  AB_LAUNCH_CHECK("tc gemm_kernel");
  return AB_OK;
}

}  // namespace tc
}  // namespace ab
