// Tensor-core GEMM core for sm_100a (tcgen05 + TMA), shared by the batched
// HLR data passes and the plain checking entry point:
//
//   C[M x N] = sum_p A_p[M x K] * B_p[N x K]^T     A, B bf16, row-major (K-major)
//
// "Parts" let one operand be a sum of bf16 slices of an FP32 matrix: with
// PA = 3 the A operand is hi + mid + lo and B is shared by the three
// products, so an FP32 matrix times a bf16 matrix is computed to FP32
// accuracy on the bf16 tensor pipe.  At most one of PA, PB is above 1.
//
// Where each 64-wide K step of an operand lives is given by an Addr: the
// tensor-map coordinate of (K step kb, part p, tile start r) is
//   x = kb * x_kb + p * x_p,   y = r + kb * y_kb + p * y_p.
// Row-major [rows][K] operands use x_kb = 64 (parts x_p elements apart);
// K-blocked operands ([K/64][parts][rows][64], one contiguous 16 KB box per
// tile) use x = 0 and y_kb, y_p row offsets.
//
// Persistent kernel: one CTA per SM walks the 128 x BN output tiles
// (tile = blockIdx.x + i * gridDim.x; tile -> (m fastest, n, split)).
// Six warps:
//   warp 0 lane 0  TMA producer: per K step PA 128x64 A tiles and PB BNx64 B
//                  tiles, 128-byte swizzled, into a STAGES-deep ring;
//   warp 1 lane 0  MMA issuer: tcgen05.mma.cta_group::1.kind::f16 (M = 128,
//                  N = BN, K = 16) into one of two FP32 accumulators in
//                  tensor memory, so the next tile's MMAs overlap the
//                  previous tile's epilogue;
//   warps 2..      epilogue (Epi::kWarps warps, a multiple of 4): warp w reads
//                  TMEM lanes 32(w%4)..+31 (one output row per thread); the
//                  kWarps/4 warps of one lane quarter split the columns into
//                  groups; 32 columns at a time come out with tcgen05.ld and
//                  go to the epilogue functor.
// Every mbarrier wait is bounded (clock-based); on expiry the kernel records
// AB_ERR_TIMEOUT in *err, stops issuing, waits (bounded) for its outstanding
// copies and MMAs, frees its tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ab {
namespace tc {

constexpr int BM = 128;
constexpr int BK = 64;                      // 64 bf16 = one 128-byte swizzle row
// threads of a launch whose epilogue has `epi_warps` warps (a multiple of 4)
__host__ __device__ constexpr int threads_for(int epi_warps) { return 64 + 32 * epi_warps; }
constexpr long long WAIT_CYCLES = 4000000000LL;   // ~2 s at 2 GHz
constexpr int SMEM_BUDGET = 232448;                // 227 KB opt-in per block

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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the phase with the given parity; false once `limit`
// cycles have passed without it.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, long long limit) {
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
    if (clock64() - t0 > limit) return false;
  }
}

// The kernels' wait: about two seconds at the SM clock.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, WAIT_CYCLES);
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

// Named barrier over the epilogue warps.
__device__ __forceinline__ void epi_sync(int nthreads) { asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory"); }
// The same barrier returning the OR of every participating thread's flag.
__device__ __forceinline__ bool epi_sync_or(int nthreads, bool flag) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)flag), "r"(nthreads)
      : "memory");
  return r != 0;
}

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

// The same load in two halves: issue (the registers fill asynchronously) and
// wait (tcgen05.wait::ld, with the registers passed through so that every
// use of them comes after it).  At most one load per thread is outstanding
// where these are used.
#define AB_R32(r) "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), \
    "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]),      \
    "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),    \
    "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
__device__ __forceinline__ void tmem_ld32_issue(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait32(uint32_t* r) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" : AB_R32(r) : : "memory");
}
#undef AB_R32
#define AB_R16(r) "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), \
    "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
// 16 columns: the same pair of halves.
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait16(uint32_t* r) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" : AB_R16(r) : : "memory");
}
#undef AB_R16

// The epilogue's walk over the 32-column chunks [cbeg, cend) of one
// accumulator (taddr: this warp's lane quarter at column 0): the next
// chunk's tensor-memory load is issued before the current chunk goes to the
// epilogue functor, so its latency hides behind that work.  have = false
// hands zeros to the functor (an empty split or a failed wait); all
// conditions are uniform over the warp, as tcgen05.ld requires.
template <class Epi>
__device__ __forceinline__ void epi_columns(Epi& e, uint32_t taddr, int cbeg, int cend, bool have, int row,
                                            int col_base, bool row_ok) {
  if (cbeg >= cend) return;
  float v[32];
  if (!have) {
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = 0.0f;
    for (int c0 = cbeg; c0 < cend; c0 += 32) e.rows(row, col_base + c0, v, row_ok);
    return;
  }
  uint32_t a[32], b[32];
  tmem_ld32_issue(taddr + (uint32_t)cbeg, a);
  tmem_wait32(a);
  for (int c0 = cbeg;; c0 += 64) {
    const bool m1 = c0 + 32 < cend, m2 = c0 + 64 < cend;
    if (m1) tmem_ld32_issue(taddr + (uint32_t)(c0 + 32), b);
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(a[k]);
    e.rows(row, col_base + c0, v, row_ok);
    if (!m1) break;
    tmem_wait32(b);
    if (m2) tmem_ld32_issue(taddr + (uint32_t)(c0 + 64), a);
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(b[k]);
    e.rows(row, col_base + c0 + 32, v, row_ok);
    if (!m2) break;
    tmem_wait32(a);
  }
}

struct Addr {
  int x_kb, x_p, y_kb, y_p;
};

// Problem shape as the kernel sees it.  K is the reduction length of one
// part.  Each split covers k_split elements of K (a multiple of BK); the
// host makes every split non-empty.
struct Shape {
  int M, N, K;
  int k_split;
  Addr a, b;
  int m_tiles, n_tiles, splits;
};

template <int BN, int PA, int PB, int EPI_SMEM>
struct Cfg {
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN in {32, 64, ..., 256}");
  static_assert(PA >= 1 && PB >= 1 && (PA == 1 || PB == 1), "one operand may have parts");
  static constexpr int P = PA > PB ? PA : PB;
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = PA * A_BYTES + PB * B_BYTES;
  static constexpr int FIXED = 1024 + 512 + EPI_SMEM;   // alignment slack, barriers, epilogue
  static constexpr int FIT = (SMEM_BUDGET - FIXED) / STAGE_BYTES;
  static constexpr int STAGES = FIT > 8 ? 8 : FIT;
  static_assert(STAGES >= 2, "tile does not fit two stages in shared memory");
  static constexpr int ACC_COLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  static constexpr int TMEM_COLS = 2 * ACC_COLS;          // two accumulators
  static constexpr int BAR_OFFSET = STAGES * STAGE_BYTES;
  static constexpr int EPI_OFFSET = BAR_OFFSET + 512;
  static constexpr int SMEM_BYTES = EPI_OFFSET + EPI_SMEM + 1024;
};

// The kernel.  Epi must provide (called by the epilogue threads only;
// etid = 0..32*kWarps-1, row = this thread's output row, cg = its column
// group, 0..kWarps/4-1):
//   static constexpr int kSmem, kWarps;
//   __device__ void begin(int m_tile, int n_tile, int split, char* smem, int etid);
//   __device__ void rows(int row, int col0, const float* v32, bool row_ok);
//   __device__ void end(int m_tile, int n_tile, int split, int row, bool row_ok, int cg);
// begin() may fill shared memory; a named barrier over the epilogue warps
// separates begin() from rows() and end() from the next tile's begin().
template <int BN, int PA, int PB, class Epi>
__global__ void __launch_bounds__(threads_for(Epi::kWarps), 1)
gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, Shape sh, Epi epi,
            int* __restrict__ err) {
  using C = Cfg<BN, PA, PB, Epi::kSmem>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* ring = base;
  uint64_t* full = reinterpret_cast<uint64_t*>(base + C::BAR_OFFSET);
  uint64_t* empty = full + C::STAGES;
  uint64_t* acc_full = empty + C::STAGES;   // [2] MMA -> epilogue
  uint64_t* acc_empty = acc_full + 2;       // [2] epilogue -> MMA
  uint64_t* drain = acc_empty + 2;          // MMA issuer's final completion
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);
  int* epi_fail = fail + 1;
  char* epi_smem = reinterpret_cast<char*>(base + C::EPI_OFFSET);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total = sh.m_tiles * sh.n_tiles * sh.splits;
  const int kb_all = (sh.K + BK - 1) / BK;
  const int kb_per_split = sh.k_split / BK;

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

  int issued = 0;   // TMA stages issued (producer), for the drain on failure
  if (warp == 0) {
    if (lane == 0) {
      int g = 0;   // global K-step counter across tiles (ring position)
      for (int t = blockIdx.x; t < total && !*(volatile int*)fail; t += gridDim.x) {
        const int mt = t % sh.m_tiles, nt = (t / sh.m_tiles) % sh.n_tiles, sp = t / (sh.m_tiles * sh.n_tiles);
        const int kb0 = sp * kb_per_split, kb1 = min(kb_all, kb0 + kb_per_split);
        for (int kb = kb0; kb < kb1; ++kb, ++g) {
          const int s = g % C::STAGES;
          const uint32_t ph = (g / C::STAGES) & 1;
          if (g >= C::STAGES && !mbar_wait(&empty[s], ph ^ 1)) { *fail = 1; break; }
          if (*(volatile int*)fail) break;
          unsigned char* a = ring + s * C::STAGE_BYTES;
          unsigned char* b = a + PA * C::A_BYTES;
          mbar_expect_tx(&full[s], C::STAGE_BYTES);
#pragma unroll
          for (int p = 0; p < PA; ++p)
            tma_load_2d(a + p * C::A_BYTES, &ta, &full[s], kb * sh.a.x_kb + p * sh.a.x_p,
                        mt * BM + kb * sh.a.y_kb + p * sh.a.y_p);
#pragma unroll
          for (int p = 0; p < PB; ++p)
            tma_load_2d(b + p * C::B_BYTES, &tb, &full[s], kb * sh.b.x_kb + p * sh.b.x_p,
                        nt * BN + kb * sh.b.y_kb + p * sh.b.y_p);
          ++issued;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = make_idesc(BN);
      int g = 0, i = 0;
      for (int t = blockIdx.x; t < total; t += gridDim.x, ++i) {
        const int sp = t / (sh.m_tiles * sh.n_tiles);
        const int kb0 = sp * kb_per_split, kb1 = min(kb_all, kb0 + kb_per_split);
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
        mma_commit(&acc_full[ab]);   // arrives when this tile's MMAs have completed
      }
      // every MMA this thread issued has completed before tensor memory is freed
      mma_commit(drain);
      if (!mbar_wait(drain, 0)) *fail = 1;
    }
  } else {
    // epilogue warps 2 .. 2+kWarps-1
    constexpr int EW = Epi::kWarps;
    static_assert(EW % 4 == 0 && EW >= 4, "epilogue warps: a multiple of 4");
    constexpr int GROUPS = EW / 4;
    static_assert(BN % (32 * GROUPS) == 0, "column groups of whole 32-column chunks");
    constexpr int GCOLS = BN / GROUPS;
    const int q = warp & 3;                 // TMEM lane quarter this warp may access
    const int cg = (warp - 2) >> 2;         // column group
    const int etid = (warp - 2) * 32 + lane;
    Epi e(epi);                             // per-thread copy: functors may keep running sums
    int i = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++i) {
      const int mt = t % sh.m_tiles, nt = (t / sh.m_tiles) % sh.n_tiles, sp = t / (sh.m_tiles * sh.n_tiles);
      const int kb0 = sp * kb_per_split, kb1 = min(kb_all, kb0 + kb_per_split);
      const int ab = i & 1;
      e.begin(mt, nt, sp, epi_smem, etid);
      epi_sync(32 * EW);
      // warp-uniform: tcgen05.ld is a warp-collective instruction
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[ab], (i >> 1) & 1));
      fence_after();
      const bool have = __all_sync(0xffffffffu, ok && kb1 > kb0 && !*(volatile int*)fail);
      const int row = mt * BM + q * 32 + lane;
      const bool row_ok = row < sh.M;
      epi_columns(e, tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * C::ACC_COLS), cg * GCOLS,
                  (cg + 1) * GCOLS, have, row, nt * BN, row_ok);
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[ab]);
      e.end(mt, nt, sp, row, row_ok, cg);
      if (!ok || *(volatile int*)fail) { *fail = 1; *(volatile int*)epi_fail = 1; }
      epi_sync(32 * EW);
      // uniform across the epilogue warps: written only before the barrier
      if (*(volatile int*)epi_fail) break;
    }
  }
  __syncwarp();
  // drain: a producer that stopped early may still have copies in flight;
  // the last copy issued into each stage is the one still outstanding there
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
