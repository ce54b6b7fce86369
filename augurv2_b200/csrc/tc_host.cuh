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

// Number of SMs of the current device (cached per device).
int sm_count();

// Operand addressing: row-major [rows][K] with parts `pstride` elements
// apart, or K-blocked [K/64][parts][blk_rows][64].
inline Addr row_major(int pstride) { return Addr{BK, pstride, 0, 0}; }
inline Addr k_blocked(int parts, int blk_rows) { return Addr{0, 0, parts * blk_rows, blk_rows}; }

// Shape with K split into at most `splits` non-empty ranges of whole K steps.
inline Shape make_shape(int M, int N, int K, int splits, Addr a, Addr b, int bn) {
  Shape s;
  s.M = M;
  s.N = N;
  s.K = K;
  const int kb_all = (K + BK - 1) / BK;
  if (splits < 1) splits = 1;
  if (splits > kb_all) splits = kb_all;
  const int per = (kb_all + splits - 1) / splits;
  s.k_split = per * BK;
  s.splits = (kb_all + per - 1) / per;
  s.a = a;
  s.b = b;
  s.m_tiles = (M + BM - 1) / BM;
  s.n_tiles = (N + bn - 1) / bn;
  return s;
}

template <int BN, int PA, int PB, class Epi>
int launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, const Shape& sh, const Epi& epi, int* err,
                cudaStream_t st) {
  using C = Cfg<BN, PA, PB, Epi::kSmem>;
  static_assert(C::SMEM_BYTES <= SMEM_BUDGET, "GEMM tile exceeds shared memory");
  AB_CUDA(cudaFuncSetAttribute(gemm_kernel<BN, PA, PB, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               C::SMEM_BYTES));
  const long long total = (long long)sh.m_tiles * sh.n_tiles * sh.splits;
  AB_REQUIRE(total > 0 && total < (1LL << 31), AB_ERR_ARG, "GEMM tile count out of range");
  const int grid = (int)(total < sm_count() ? total : sm_count());
  gemm_kernel<BN, PA, PB, Epi><<<grid, threads_for(Epi::kWarps), C::SMEM_BYTES, st>>>(ta, tb, sh, epi, err);
  AB_LAUNCH_CHECK("tc gemm_kernel");
  return AB_OK;
}

}  // namespace tc
}  // namespace ab
