// Tensor-core GEMM core for sm_100a (tcgen05 + TMA), shared by the batched
// HLR data passes and the gradient-surrogate MLP:
//
//   C[M x N] = A[M x K] * B[N x K]^T        A, B bf16, row-major (K-major)
//
// One CTA computes one 128 x BN output tile (BN <= 256) over a K range
// (split-K via blockIdx.z).  Four warps:
//   warp 0 lane 0  TMA producer: 128x64 A tiles and BNx64 B tiles, 128-byte
//                  swizzled, into a STAGES-deep ring guarded by mbarriers;
//   warp 1 lane 0  MMA issuer: tcgen05.mma.cta_group::1.kind::f16 (M=128,
//                  N=BN, K=16) into an FP32 accumulator in tensor memory,
//                  tcgen05.commit frees each stage and finally signals done;
//   all 4 warps    epilogue: warp w reads TMEM lanes 32w..32w+31 (one output
//                  row per thread) 32 columns at a time with tcgen05.ld and
//                  hands them to the epilogue functor.
// Every mbarrier wait is bounded (clock-based); on expiry the kernel records
// AB_ERR_TIMEOUT in *err, drains its outstanding copies, frees its tensor
// memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ab {
namespace tc {

constexpr int BM = 128;
constexpr int BK = 64;                      // 64 bf16 = one 128-byte swizzle row
constexpr long long WAIT_CYCLES = 4000000000LL;   // ~2 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > WAIT_CYCLES) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t make_desc(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t make_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive fp32 columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN>
struct Cfg {
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN in {32, 64, ..., 256}");
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int STAGES = (BN >= 256) ? 4 : (BN >= 128 ? 6 : 8);
  static constexpr int TMEM_COLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  // ring + barriers + tmem slot, with 1024-byte alignment slack; the
  // epilogue's own shared memory (Epi::kSmem) follows at EPI_OFFSET
  static constexpr int EPI_OFFSET = STAGES * STAGE_BYTES + 256;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
};

// The kernel.  Epi must provide:
//   __device__ void begin(int m_tile, int n_tile, int split, char* smem_scratch)   (all threads)
//   __device__ void rows(int row, int col0, const float* v32, bool row_ok)        (all threads, per 32 cols)
//   __device__ void end(int m_tile, int n_tile, int split)                        (all threads)
template <int BN, class Epi>
__global__ void __launch_bounds__(128, 1)
gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int M, int N, int K,
            int k_split, Epi epi, int* __restrict__ err) {
  using C = Cfg<BN>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* ring = base;
  uint64_t* full = reinterpret_cast<uint64_t*>(base + C::STAGES * C::STAGE_BYTES);
  uint64_t* empty = full + C::STAGES;
  uint64_t* done = empty + C::STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kb0 = (blockIdx.z * k_split) / BK;
  const int kb1 = min((K + BK - 1) / BK, ((blockIdx.z + 1) * k_split) / BK);
  const int nkb = max(0, kb1 - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    *fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)C::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  epi.begin(blockIdx.x, blockIdx.y, blockIdx.z, reinterpret_cast<char*>(base + C::EPI_OFFSET));

  int issued = 0;   // TMA stages issued (producer)
  if (threadIdx.x == 0) {
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % C::STAGES;
      const uint32_t ph = (kb / C::STAGES) & 1;
      if (kb >= C::STAGES && !mbar_wait(&empty[s], ph ^ 1)) { *fail = 1; break; }
      if (*(volatile int*)fail) break;
      unsigned char* a = ring + s * C::STAGE_BYTES;
      unsigned char* b = a + C::A_BYTES;
      mbar_expect_tx(&full[s], C::STAGE_BYTES);
      tma_load_2d(a, &ta, &full[s], (kb0 + kb) * BK, m0);
      tma_load_2d(b, &tb, &full[s], (kb0 + kb) * BK, n0);
      ++issued;
    }
  } else if (threadIdx.x == 32) {
    const uint32_t idesc = make_idesc(BN);
    int kb = 0;
    for (; kb < nkb; ++kb) {
      const int s = kb % C::STAGES;
      const uint32_t ph = (kb / C::STAGES) & 1;
      if (!mbar_wait(&full[s], ph)) { *fail = 1; break; }
      if (*(volatile int*)fail) break;
      fence_after();
      const uint64_t ad = make_desc(ring + s * C::STAGE_BYTES);
      const uint64_t bd = make_desc(ring + s * C::STAGE_BYTES + C::A_BYTES);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk)
        mma_bf16(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
      mma_commit(&empty[s]);
    }
    mma_commit(done);   // arrives when every issued MMA has completed
  }
  __syncwarp();
  // epilogue
  bool ok = mbar_wait(done, 0);
  fence_after();
  if (!ok) *fail = 1;
  const bool have = nkb > 0 && ok && !*(volatile int*)fail;
  const int row = m0 + warp * 32 + lane;
  for (int c0 = 0; c0 < BN; c0 += 32) {
    float v[32];
    if (have) {
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
    } else {
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = 0.0f;
    }
    epi.rows(row, n0 + c0, v, row < M);
  }
  epi.end(blockIdx.x, blockIdx.y, blockIdx.z);
  // drain: a producer that stopped early still has copies in flight
  if (threadIdx.x == 0 && *(volatile int*)fail) {
    for (int kb = 0; kb < issued; ++kb) mbar_wait(&full[kb % C::STAGES], (kb / C::STAGES) & 1);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)C::TMEM_COLS)
                 : "memory");
  }
  if (threadIdx.x == 0 && *(volatile int*)fail && err) atomicExch(err, 3 /* AB_ERR_TIMEOUT */);
}

}  // namespace tc
}  // namespace ab
