// Grouped variant of the tensor-core GEMM core: ONE persistent launch walks
// the output tiles of many independent problems (model instances of uneven
// size), each with its own tensor maps, shape, output-tile width and
// epilogue parameters, read from tables in device memory:
//
//   probs[i]   GProblem: operand tensor maps, Shape, output-tile width bn_i
//              (<= BN, a multiple of 32) and tile0_i, the index of the
//              problem's first tile in the launch's tile order;
//   epis[i]    the epilogue functor of problem i (its parameter fields; the
//              per-thread fields are reset by begin());
//   head       {n, total}: problems in use (the first n of the tables) and
//              their tiles.  Both live in device memory, so a captured CUDA
//              graph of the launch picks up a new set of problems without
//              being captured again.
//
// Tile t belongs to the problem i with tile0_i <= t < tile0_{i+1} (binary
// search in a shared-memory copy of the tile0 column); inside a problem the
// order is that of gemm_kernel (m fastest, then n, then split), so a
// problem's partial results are bit-identical to its own launch of
// gemm_kernel with the same Shape and tile width.  Roles, pipeline, bounded
// waits and the failure drain are gemm_kernel's.  The tensor maps are
// written by host copies before the launch; the producer issues a tensormap
// acquire fence for each problem's maps before their first use.
#pragma once
#include "tc_gemm.cuh"

namespace ab {
namespace tc {

constexpr int GROUP_MAX = 256;   // problems per grouped launch

struct alignas(64) GProblem {
  CUtensorMap ta;   // A operand: BM-row boxes
  CUtensorMap tb;   // B operand: bn-row boxes
  Shape sh;
  int bn;           // output-tile width of this problem (32..BN, a multiple of 32)
  int tile0;        // first tile of this problem
};

struct GHead {
  int n, total;
};

__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(m))
               : "memory");
}

// Problem owning tile t: the last i < n with tile0[i] <= t.
__device__ __forceinline__ int group_find(const int* tile0, int n, int t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile0[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int BN, int PA, int PB, class Epi>
struct GCfg {
  static constexpr int kTableBytes = 4 * GROUP_MAX;
  using C = Cfg<BN, PA, PB, Epi::kSmem + kTableBytes>;
};

template <int BN, int PA, int PB, class Epi>
__global__ void __launch_bounds__(threads_for(Epi::kWarps), 1)
grouped_gemm_kernel(const GProblem* __restrict__ probs, const Epi* __restrict__ epis, const GHead* __restrict__ head,
                    int* __restrict__ err) {
  using C = typename GCfg<BN, PA, PB, Epi>::C;
  const int n = head->n, total = head->total;
  if (n <= 0 || (int)blockIdx.x >= total) return;   // uniform over the CTA: nothing to do
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* ring = base;
  uint64_t* full = reinterpret_cast<uint64_t*>(base + C::BAR_OFFSET);
  uint64_t* empty = full + C::STAGES;
  uint64_t* acc_full = empty + C::STAGES;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);
  int* epi_fail = fail + 1;
  char* epi_smem = reinterpret_cast<char*>(base + C::EPI_OFFSET);
  int* tile0 = reinterpret_cast<int*>(epi_smem + Epi::kSmem);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ng = n < GROUP_MAX ? n : GROUP_MAX;
  for (int i = threadIdx.x; i < ng; i += blockDim.x) tile0[i] = probs[i].tile0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int b = 0; b < 2; ++b) { mbar_init(&acc_full[b], 1); mbar_init(&acc_empty[b], Epi::kWarps); }
    mbar_init(drain, 1);
    *fail = 0;
    *epi_fail = 0;
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

  int issued = 0;
  if (warp == 0) {
    if (lane == 0) {
      int g = 0, last = -1;
      for (int t = blockIdx.x; t < total && !*(volatile int*)fail; t += gridDim.x) {
        const int pi = group_find(tile0, ng, t);
        const GProblem* P = probs + pi;
        if (pi != last) {
          tensormap_acquire(&P->ta);
          tensormap_acquire(&P->tb);
          last = pi;
        }
        const Shape sh = P->sh;
        const int lt = t - tile0[pi];
        const int mt = lt % sh.m_tiles, nt = (lt / sh.m_tiles) % sh.n_tiles, sp = lt / (sh.m_tiles * sh.n_tiles);
        const int kb_all = (sh.K + BK - 1) / BK, kb_per_split = sh.k_split / BK;
        const int kb0 = sp * kb_per_split, kb1 = min(kb_all, kb0 + kb_per_split);
        const int bn = P->bn;
        const uint32_t bytes = (uint32_t)(PA * C::A_BYTES + PB * bn * BK * 2);
        for (int kb = kb0; kb < kb1; ++kb, ++g) {
          const int s = g % C::STAGES;
          const uint32_t ph = (g / C::STAGES) & 1;
          if (g >= C::STAGES && !mbar_wait(&empty[s], ph ^ 1)) { *fail = 1; break; }
          if (*(volatile int*)fail) break;
          unsigned char* a = ring + s * C::STAGE_BYTES;
          unsigned char* b = a + PA * C::A_BYTES;
          mbar_expect_tx(&full[s], bytes);
#pragma unroll
          for (int p = 0; p < PA; ++p)
            tma_load_2d(a + p * C::A_BYTES, &P->ta, &full[s], kb * sh.a.x_kb + p * sh.a.x_p,
                        mt * BM + kb * sh.a.y_kb + p * sh.a.y_p);
#pragma unroll
          for (int p = 0; p < PB; ++p)
            tma_load_2d(b + p * C::B_BYTES, &P->tb, &full[s], kb * sh.b.x_kb + p * sh.b.x_p,
                        nt * bn + kb * sh.b.y_kb + p * sh.b.y_p);
          ++issued;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int g = 0, i = 0;
      for (int t = blockIdx.x; t < total; t += gridDim.x, ++i) {
        const int pi = group_find(tile0, ng, t);
        const GProblem* P = probs + pi;
        const Shape sh = P->sh;
        const int lt = t - tile0[pi];
        const int sp = lt / (sh.m_tiles * sh.n_tiles);
        const int kb_all = (sh.K + BK - 1) / BK, kb_per_split = sh.k_split / BK;
        const int kb0 = sp * kb_per_split, kb1 = min(kb_all, kb0 + kb_per_split);
        const uint32_t idesc = make_idesc(P->bn);
        const int ab = i & 1;
        if (i >= 2 && !mbar_wait(&acc_empty[ab], ((i >> 1) - 1) & 1)) { *fail = 1; break; }
        if (*(volatile int*)fail) break;
        fence_after();
        const uint32_t d = tmem + (uint32_t)(ab * C::ACC_COLS);
        bool bad = false;
        for (int kb = kb0; kb < kb1; ++kb, ++g) {
          const int s = g % C::STAGES;
          const uint32_t ph = (g / C::STAGES) & 1;
          if (!mbar_wait(&full[s], ph)) { *fail = 1; bad = true; break; }
          if (*(volatile int*)fail) { bad = true; break; }
          fence_after();
          unsigned char* a = ring + s * C::STAGE_BYTES;
          unsigned char* b = a + PA * C::A_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
#pragma unroll
            for (int p = 0; p < C::P; ++p) {
              const uint64_t ad = make_desc(a + (PA > 1 ? p : 0) * C::A_BYTES) + 2 * kk;
              const uint64_t bd = make_desc(b + (PB > 1 ? p : 0) * C::B_BYTES) + 2 * kk;
              mma_bf16(d, ad, bd, idesc, (kb > kb0 || kk > 0 || p > 0) ? 1u : 0u);
            }
          }
          mma_commit(&empty[s]);
        }
        if (bad) break;
        mma_commit(&acc_full[ab]);
      }
      mma_commit(drain);
      if (!mbar_wait(drain, 0)) *fail = 1;
    }
  } else {
    constexpr int EW = Epi::kWarps;
    static_assert(EW % 4 == 0 && EW >= 4, "epilogue warps: a multiple of 4");
    constexpr int GROUPS = EW / 4;
    static_assert(BN % (32 * GROUPS) == 0, "column groups of whole 32-column chunks");
    constexpr int GCOLS = BN / GROUPS;
    const int q = warp & 3;
    const int cg = (warp - 2) >> 2;
    const int etid = (warp - 2) * 32 + lane;
    int i = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++i) {
      const int pi = group_find(tile0, ng, t);
      const GProblem* P = probs + pi;
      const Shape sh = P->sh;
      const int lt = t - tile0[pi];
      const int mt = lt % sh.m_tiles, nt = (lt / sh.m_tiles) % sh.n_tiles, sp = lt / (sh.m_tiles * sh.n_tiles);
      const int kb_all = (sh.K + BK - 1) / BK, kb_per_split = sh.k_split / BK;
      const int kb0 = sp * kb_per_split, kb1 = min(kb_all, kb0 + kb_per_split);
      const int bn = P->bn;
      const int ab = i & 1;
      Epi e = epis[pi];
      e.begin(mt, nt, sp, epi_smem, etid);
      epi_sync(32 * EW);
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[ab], (i >> 1) & 1));
      fence_after();
      const bool have = __all_sync(0xffffffffu, ok && kb1 > kb0 && !*(volatile int*)fail);
      const int row = mt * BM + q * 32 + lane;
      const bool row_ok = row < sh.M;
      epi_columns(e, tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * C::ACC_COLS), cg * GCOLS,
                  min((cg + 1) * GCOLS, bn), have, row, nt * bn, row_ok);
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[ab]);
      e.end(mt, nt, sp, row, row_ok, cg);
      if (!ok || *(volatile int*)fail) { *fail = 1; *(volatile int*)epi_fail = 1; }
      epi_sync(32 * EW);
      if (*(volatile int*)epi_fail) break;
    }
  }
  __syncwarp();
  if (threadIdx.x == 0 && *(volatile int*)fail) {
    for (int g = max(0, issued - C::STAGES); g < issued; ++g)
      mbar_wait(&full[g % C::STAGES], (g / C::STAGES) & 1);
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
