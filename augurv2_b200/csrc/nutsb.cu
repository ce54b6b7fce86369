// Batched NUTS: C chains of the reference's No-U-Turn sampler
// (h_augur_mcmc_nuts / h_augur_nuts_build_tree / h_augur_nuts_update_s,
// cbits/augur_mcmclib.h:575-776) advanced together, with every leaf's log
// density and gradient supplied by one batched evaluation for all chains
// (the tensor-core HLR pass).
//
// Each chain is a resumable state machine kept in device memory.  A call of
// ab_nutsb_advance runs every chain's tree walk (one CTA per chain) until the
// chain reaches its next leaf: it performs the leaf's first half kick and
// drift, leaves the new position in `thprop` and stops.  The caller then
// evaluates log density and gradient at every chain's `thprop`, and the next
// advance finishes the leaf (second half kick, slice tests) and walks on.
// So every chain needs exactly one gradient per round and the batched pass
// is always full; a chain whose tree terminates records its draw and starts
// its next iteration in the same call (chains run asynchronously, each with
// its own iteration counter).
//
// The walk is the reference's, quirks included: a post-order walk of the
// doubling tree over an explicit frame stack; subtree end points pushed
// only by j == 1 subtrees; the proposal of a doubling replaces the
// iteration's draw only if the last doubling accepts it; augur_min on
// unsigned values when biasing the top-level choice.  The leapfrog of a leaf
// uses the gradient already known at its start point (the reference
// re-evaluates it; the value is the same).  Positions, momenta and
// gradients are FP32; the slice variable, the Hamiltonians and the U-turn
// dot products are FP64.  Random streams match the per-chain sampler:
// momenta (seed, chain * P + j, iteration, MOM | comp << 8), one normal
// each; the slice, direction and selection uniforms from the sequential
// stream (seed, chain, iteration, NUTS | comp << 8).
#include <math.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "common.cuh"
#include "philox.cuh"

namespace ab {
namespace {

constexpr int NB_THREADS = 128;
constexpr int NB_STK = 16;        // stack entries (cbits/augur_blkstk.h:26)
constexpr int NB_FRAMES = 24;
constexpr int NB_GUARD = 100000;  // walk steps per call before giving up (error)

enum { M_START = 0, M_DOUBLING = 1, M_WALK = 2, M_LEAF = 3 };

struct Frame {
  int j, phase, ln, ls;
};

struct ChainState {
  int mode, sp, n, jd, s, dir, rn, rs, f_cpy, leaves, overflow;
  int tp_h, ts_h, ms_h;
  uint32_t iter, h_pos;
  int ndraws, last_depth, last_leaves, error, divergences, div_flag;
  float stepsize;
  double logu, ll0, sel_ll, depth_sum;
  Frame fr[NB_FRAMES];
};

__device__ __forceinline__ double block_dot(const float* a, const float* b, int P, double* red) {
  double s = 0.0;
  for (int j = threadIdx.x; j < P; j += blockDim.x) s += (double)a[j] * (double)b[j];
  return block_sum_f64(s, red);
}

__device__ __forceinline__ double block_diff_dot(const float* a, const float* b, const float* m, int P,
                                                 double* red) {
  double s = 0.0;
  for (int j = threadIdx.x; j < P; j += blockDim.x) s += ((double)a[j] - (double)b[j]) * (double)m[j];
  return block_sum_f64(s, red);
}

__device__ __forceinline__ void copy_vec(float* dst, const float* src, int P) {
  for (int j = threadIdx.x; j < P; j += blockDim.x) dst[j] = src[j];
}

}  // namespace

// Everything the advance kernel touches, by chain.
struct NutsbDev {
  int C, P, max_depth, hist_cap;
  int standard;               // 0: the reference's selection (quirks), 1: Hoffman & Gelman's
  uint64_t seed;
  uint32_t comp;
  float eps;
  ChainState* st;
  float *th0, *g0, *thm, *gm, *thp, *gp, *thprop, *gprop, *mm, *mp, *sel, *selg;
  float *tp, *tpg, *ts, *ms;  // stacks [C][NB_STK][P]
  double* tpll;               // [C][NB_STK]
  const double* logp_new;     // [C] at thprop (from the caller's pass)
  const float* g_new;         // [C][P]
  float* hist;                // [C][hist_cap][P] draws
  int* hist_depth;            // [C][hist_cap] tree depth of each draw
};

namespace {

// One chain's walk to its next leaf (one CTA of NB_THREADS threads), shared
// by the per-sampler and the grouped launch.
__device__ __forceinline__ void advance_chain(const NutsbDev& dv, const int c) {
  __shared__ ChainState S;
  __shared__ double red[33];
  __shared__ double dsh[2];
  const int P = dv.P, tid = threadIdx.x;
  if (tid == 0) S = dv.st[c];
  __syncthreads();
  const size_t o = (size_t)c * P;
  float *th0 = dv.th0 + o, *g0 = dv.g0 + o, *thm = dv.thm + o, *gm = dv.gm + o, *thp = dv.thp + o,
        *gp = dv.gp + o, *thprop = dv.thprop + o, *gprop = dv.gprop + o, *mm = dv.mm + o, *mp = dv.mp + o,
        *sel = dv.sel + o, *selg = dv.selg + o;
  float* tp = dv.tp + (size_t)c * NB_STK * P;
  float* tpg = dv.tpg + (size_t)c * NB_STK * P;
  float* ts = dv.ts + (size_t)c * NB_STK * P;
  float* ms = dv.ms + (size_t)c * NB_STK * P;
  double* tpll = dv.tpll + (size_t)c * NB_STK;

  // next uniform of the chain's sequential stream (thread 0 draws; all read)
  auto draw_u = [&]() -> double {
    __syncthreads();
    if (tid == 0) {
      Stream h = make_stream(dv.seed, (uint32_t)c, S.iter, TAG_NUTS | (dv.comp << 8));
      h.pos = S.h_pos;
      dsh[0] = h.uniform();
      S.h_pos = h.pos;
    }
    __syncthreads();
    return dsh[0];
  };
  // stack push: returns the slot written (all threads)
  auto push_slot = [&](int* head) -> int {
    __syncthreads();
    int hd = *head + 1;
    if (hd >= NB_STK) hd = NB_STK - 1;
    __syncthreads();
    if (tid == 0) {
      if (*head + 1 >= NB_STK) S.overflow = 1;
      *head = hd;
    }
    __syncthreads();
    return hd;
  };
  auto pop_slot = [&](int* head) -> int {
    __syncthreads();
    const int h = *head;
    __syncthreads();
    if (tid == 0) *head = h - 1;
    __syncthreads();
    return h < 0 ? 0 : h;
  };
  auto top = [&](int head) -> int { return head < 0 ? 0 : head; };
  // h_augur_nuts_update_s: s && (tp - tm).mp >= 0 && (tp - tm).mm >= 0
  auto update_s = [&](int s, const float* tpv, const float* mpv, const float* tmv, const float* mmv) -> int {
    if (s != 1) return 0;
    const double d1 = block_diff_dot(tpv, tmv, mpv, P, red);
    const double d2 = block_diff_dot(tpv, tmv, mmv, P, red);
    return (d1 >= 0.0 && d2 >= 0.0) ? 1 : 0;
  };

  for (int guard = 0; guard < NB_GUARD; ++guard) {
    // snapshot of the scalar state: every thread reads it between two
    // barriers, so thread 0's updates later in this step cannot race the reads
    __syncthreads();
    const int mode = S.mode, sp = S.sp, rn = S.rn, rs = S.rs, dir = S.dir, n_s = S.n, jd_s = S.jd;
    const float stepsize = S.stepsize;
    Frame F;
    F.j = F.phase = F.ln = F.ls = 0;
    if (sp >= 0 && sp < NB_FRAMES) F = S.fr[sp];
    __syncthreads();
    if (mode == M_LEAF) {
      // finish the leaf: the caller evaluated logp and gradient at thprop
      float* mom = dir == 0 ? mm : mp;
      const float hs = 0.5f * stepsize;
      for (int j = tid; j < P; j += blockDim.x) {
        const float g = dv.g_new[o + j];
        gprop[j] = g;
        mom[j] += hs * g;
      }
      const double llp = dv.logp_new[c];
      const int slot = push_slot(&S.tp_h);
      copy_vec(tp + (size_t)slot * P, thprop, P);
      copy_vec(tpg + (size_t)slot * P, gprop, P);
      const double ke = block_dot(mom, mom, P, red);
      if (tid == 0) {
        tpll[slot] = llp;
        S.leaves += 1;
        const double ll = llp - 0.5 * ke;
        S.rn = S.logu <= ll ? 1 : 0;
        S.rs = S.logu < 1000.0 + ll ? 1 : 0;
        if (!S.rs) S.div_flag = 1;   // outside the slice by more than deltaMax
        S.sp -= 1;
        S.mode = M_WALK;
      }
      continue;
    }
    if (mode == M_START) {
      // a new iteration at th0 (log density ll0, gradient g0 known)
      for (int j = tid; j < P; j += blockDim.x) {
        Stream s = make_stream(dv.seed, (uint32_t)c * (uint32_t)P + j, S.iter, TAG_MOM | (dv.comp << 8));
        const float m0 = (float)s.normal();
        mm[j] = m0;
        mp[j] = m0;
        thm[j] = th0[j];
        thp[j] = th0[j];
        gm[j] = g0[j];
        gp[j] = g0[j];
      }
      const double m2 = block_dot(mm, mm, P, red);
      if (tid == 0) {
        Stream h = make_stream(dv.seed, (uint32_t)c, S.iter, TAG_NUTS | (dv.comp << 8));
        const double e = -1.0 * log(h.uniform());
        S.h_pos = h.pos;
        S.logu = S.ll0 - 0.5 * m2 - e;
        S.n = 1;
        S.jd = 0;
        S.s = 1;
        S.f_cpy = 0;
        S.leaves = 0;
        S.overflow = 0;
        S.tp_h = -1;
        S.ts_h = -1;
        S.ms_h = -1;
        S.mode = M_DOUBLING;
      }
      continue;
    }
    if (mode == M_DOUBLING) {
      const double u = draw_u();
      if (tid == 0) {
        if (!dv.standard) S.f_cpy = 0;   // the reference keeps only the last doubling's pick
        S.ts_h = -1;
        S.ms_h = -1;
        S.dir = u < 0.5 ? 0 : 1;
        S.stepsize = S.dir == 0 ? -dv.eps : dv.eps;
        S.sp = 0;
        S.fr[0].j = S.jd;
        S.fr[0].phase = 0;
      }
      __syncthreads();
      const bool minus = S.dir == 0;
      copy_vec(thprop, minus ? thm : thp, P);
      copy_vec(gprop, minus ? gm : gp, P);
      if (tid == 0) S.mode = M_WALK;
      continue;
    }
    // ---- M_WALK: one step of the post-order walk
    if (sp >= NB_FRAMES - 1) {
      if (tid == 0) S.error = 2;   // deeper than the frame stack (max_depth is checked by the host)
      break;
    }
    if (sp >= 0) {
      if (F.j == 0) {
        // leaf: half kick with the known gradient, drift; then wait for the
        // caller's evaluation at the new thprop
        float* mom = dir == 0 ? mm : mp;
        const float st = stepsize, hs = 0.5f * stepsize;
        for (int j = tid; j < P; j += blockDim.x) {
          const float mv = mom[j] + hs * gprop[j];
          mom[j] = mv;
          thprop[j] += st * mv;
        }
        __syncthreads();
        if (tid == 0) S.mode = M_LEAF;
        __syncthreads();
        break;
      }
      if (F.phase == 0) {
        if (tid == 0) {
          S.fr[sp].phase = 1;
          S.fr[sp + 1].j = F.j - 1;
          S.fr[sp + 1].phase = 0;
          S.sp = sp + 1;
        }
        continue;
      }
      if (F.phase == 1) {
        // left subtree finished
        const int ln = rn, ls = rs;
        if (ls == 1) {
          if (F.j == 1) {
            const float* mom = dir == 0 ? mm : mp;
            const int a = push_slot(&S.ts_h);
            copy_vec(ts + (size_t)a * P, thprop, P);
            const int b = push_slot(&S.ms_h);
            copy_vec(ms + (size_t)b * P, mom, P);
          }
          __syncthreads();
          if (tid == 0) {
            S.fr[sp].ln = ln;
            S.fr[sp].ls = ls;
            S.fr[sp].phase = 2;
            S.fr[sp + 1].j = F.j - 1;
            S.fr[sp + 1].phase = 0;
            S.sp = sp + 1;
          }
        } else {
          if (tid == 0) {
            S.fr[sp].ln = ln;
            S.fr[sp].ls = ls;
            S.rn = ln;
            S.rs = ls;
            S.sp = sp - 1;
          }
        }
        continue;
      }
      // phase 2: right subtree finished (rn, rs)
      const int p1 = pop_slot(&S.tp_h);
      const int p2 = pop_slot(&S.tp_h);
      const double bias = ((double)rn) / (F.ln + rn);
      const double uu = draw_u();
      const int src = (uu < bias) ? p1 : p2;
      const int dst = push_slot(&S.tp_h);
      if (src != dst) {
        copy_vec(tp + (size_t)dst * P, tp + (size_t)src * P, P);
        copy_vec(tpg + (size_t)dst * P, tpg + (size_t)src * P, P);
      }
      __syncthreads();
      if (tid == 0 && src != dst) tpll[dst] = tpll[src];
      const int ln = F.ln + rn;
      const int th_slot = top(S.ts_h), mo_slot = top(S.ms_h);
      const float* mom = dir == 0 ? mm : mp;
      int ls;
      if (dir == 0)
        ls = update_s(rs, ts + (size_t)th_slot * P, ms + (size_t)mo_slot * P, thprop, mom);
      else
        ls = update_s(rs, thprop, mom, ts + (size_t)th_slot * P, ms + (size_t)mo_slot * P);
      if (F.j > 1) {
        pop_slot(&S.ts_h);
        pop_slot(&S.ms_h);
      }
      __syncthreads();
      if (tid == 0) {
        S.fr[sp].ln = ln;
        S.fr[sp].ls = ls;
        S.rn = ln;
        S.rs = ls;
        S.sp = sp - 1;
      }
      continue;
    }
    // ---- the doubling's tree is complete: outer loop body (:744-774)
    {
      const bool minus = dir == 0;
      copy_vec(minus ? thm : thp, thprop, P);
      copy_vec(minus ? gm : gp, gprop, P);
      const int pp = pop_slot(&S.tp_h);
      if (rs == 1) {
        double bias;
        if (dv.standard) {
          bias = fmin(1.0, ((double)rn) / n_s);
        } else {
          const unsigned ratio = (unsigned)(((double)rn) / n_s);   // augur_min on unsigned
          bias = (double)(ratio < 1u ? ratio : 1u);
        }
        if (draw_u() < bias) {
          copy_vec(sel, tp + (size_t)pp * P, P);
          copy_vec(selg, tpg + (size_t)pp * P, P);
          if (tid == 0) {
            S.sel_ll = tpll[pp];
            S.f_cpy = 1;
          }
        }
      }
      __syncthreads();
      const int s = update_s(rs, thp, mp, thm, mm);
      const int jd = jd_s + 1;
      const bool stop = s != 1 || jd >= dv.max_depth || S.overflow;
      if (tid == 0) {
        S.n += rn;
        S.s = s;
        S.jd = jd;
      }
      __syncthreads();
      if (!stop) {
        if (tid == 0) S.mode = M_DOUBLING;
        continue;
      }
      // iteration done: the draw is th0, replaced by the selected proposal (the
      // reference: the last doubling's pick only; standard: the latest pick)
      if (S.f_cpy) {
        copy_vec(th0, sel, P);
        copy_vec(g0, selg, P);
      }
      __syncthreads();
      const int k = S.ndraws;
      if (k < dv.hist_cap) {
        copy_vec(dv.hist + ((size_t)c * dv.hist_cap + k) * P, th0, P);
        if (tid == 0) dv.hist_depth[(size_t)c * dv.hist_cap + k] = jd;
      }
      __syncthreads();
      if (tid == 0) {
        if (S.f_cpy) S.ll0 = S.sel_ll;
        S.ndraws = k + 1;
        S.last_depth = jd;
        S.last_leaves = S.leaves;
        S.depth_sum += jd;
        S.divergences += S.div_flag;
        S.div_flag = 0;
        S.iter += 1;
        S.mode = M_START;
      }
      continue;
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (S.mode != M_LEAF) S.error = 1;   // the guard ran out without reaching a leaf
    dv.st[c] = S;
  }
}

__global__ void __launch_bounds__(NB_THREADS) nutsb_advance_kernel(NutsbDev dv) { advance_chain(dv, blockIdx.x); }

// Grouped advance: instance blockIdx.y of the first *n entries of tab, chain
// blockIdx.x (the grid covers the largest chain count of the group).
__global__ void __launch_bounds__(NB_THREADS) nutsg_advance_kernel(const NutsbDev* __restrict__ tab,
                                                                   const int* __restrict__ n) {
  if ((int)blockIdx.y >= *n) return;
  const NutsbDev dv = tab[blockIdx.y];
  if ((int)blockIdx.x >= dv.C) return;
  advance_chain(dv, blockIdx.x);
}

}  // namespace
}  // namespace ab

namespace ab {
namespace {
NutsbDev layout(void* mem, int C, int P, int hist_cap) {
  NutsbDev d{};
  char* p = static_cast<char*>(mem);
  auto take = [&](size_t bytes) {
    char* r = p;
    p += (bytes + 255) & ~size_t(255);
    return r;
  };
  const size_t vec = (size_t)C * P * sizeof(float);
  d.C = C;
  d.P = P;
  d.hist_cap = hist_cap;
  d.st = reinterpret_cast<ChainState*>(take((size_t)C * sizeof(ChainState)));
  float** vs[12] = {&d.th0, &d.g0, &d.thm, &d.gm, &d.thp, &d.gp, &d.thprop, &d.gprop, &d.mm, &d.mp, &d.sel, &d.selg};
  for (auto v : vs) *v = reinterpret_cast<float*>(take(vec));
  d.tp = reinterpret_cast<float*>(take(NB_STK * vec));
  d.tpg = reinterpret_cast<float*>(take(NB_STK * vec));
  d.ts = reinterpret_cast<float*>(take(NB_STK * vec));
  d.ms = reinterpret_cast<float*>(take(NB_STK * vec));
  d.tpll = reinterpret_cast<double*>(take((size_t)C * NB_STK * sizeof(double)));
  d.hist = reinterpret_cast<float*>(take((size_t)C * hist_cap * P * sizeof(float)));
  d.hist_depth = reinterpret_cast<int*>(take((size_t)C * hist_cap * sizeof(int)));
  return d;
}

__global__ void nutsb_init_kernel(NutsbDev d, const float* theta, const float* grad, const double* logp,
                                  uint32_t iter0) {
  const int c = blockIdx.x, P = d.P;
  for (int j = threadIdx.x; j < P; j += blockDim.x) {
    d.th0[(size_t)c * P + j] = theta[(size_t)c * P + j];
    d.g0[(size_t)c * P + j] = grad[(size_t)c * P + j];
  }
  if (threadIdx.x == 0) {
    ChainState s;
    memset(&s, 0, sizeof(s));
    s.mode = M_START;
    s.iter = iter0;
    s.ll0 = logp[c];
    s.tp_h = s.ts_h = s.ms_h = -1;
    d.st[c] = s;
  }
}

// Per-chain summary: [ndraws, last_depth, last_leaves, error, iter, mean depth,
// divergent iterations]
__global__ void nutsb_info_kernel(NutsbDev d, double* info) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.C) return;
  const ChainState& s = d.st[c];
  double* o = info + (size_t)c * AB_NUTSB_INFO;
  o[0] = s.ndraws;
  o[1] = s.last_depth;
  o[2] = s.last_leaves;
  o[3] = s.error;
  o[4] = s.iter;
  o[5] = s.ndraws > 0 ? s.depth_sum / s.ndraws : 0.0;
  o[6] = s.divergences;
}

// Forget the recorded draws (end of warm-up): every chain keeps its position,
// tree state and iteration counter; its draw count and depth statistics
// restart from zero.
__global__ void nutsb_reset_history_kernel(NutsbDev d) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.C) return;
  d.st[c].ndraws = 0;
  d.st[c].depth_sum = 0.0;
  d.st[c].divergences = 0;
}
}  // namespace
}  // namespace ab

using namespace ab;

// ---- C ABI ------------------------------------------------------------------
extern "C" size_t ab_nutsb_state_bytes(int C, int P, int hist_cap) {
  if (C <= 0 || P <= 0 || hist_cap < 0) return 0;
  const size_t vec = (size_t)C * P * sizeof(float);
  size_t b = 0;
  b += (size_t)C * sizeof(ChainState);
  b = (b + 255) & ~size_t(255);
  b += 12 * vec;                                   // th0 g0 thm gm thp gp thprop gprop mm mp sel selg
  b += 4 * (size_t)NB_STK * vec;                   // tp tpg ts ms
  b += (size_t)C * NB_STK * sizeof(double);        // tpll
  b += (size_t)C * hist_cap * P * sizeof(float);   // history
  b += (size_t)C * hist_cap * sizeof(int);         // history depths
  return b + 16 * 256;
}


extern "C" int ab_nutsb_init(void* mem, int C, int P, int hist_cap, const float* theta, const float* grad,
                             const double* logp, uint32_t iter0, void* stream) {
  AB_REQUIRE(mem && theta && grad && logp && C > 0 && P > 0 && hist_cap >= 0, AB_ERR_ARG, "ab_nutsb_init: bad arguments");
  AB_REQUIRE((reinterpret_cast<uintptr_t>(mem) & 255) == 0, AB_ERR_ARG, "ab_nutsb_init: state must be 256-byte aligned");
  NutsbDev d = layout(mem, C, P, hist_cap);
  nutsb_init_kernel<<<C, 128, 0, as_stream(stream)>>>(d, theta, grad, logp, iter0);
  AB_LAUNCH_CHECK("nutsb_init_kernel");
  return AB_OK;
}

extern "C" int ab_nutsb_thprop(void* mem, int C, int P, int hist_cap, float** thprop, float** hist, int** hist_depth) {
  AB_REQUIRE(mem && thprop && hist && hist_depth, AB_ERR_ARG, "ab_nutsb_thprop: null pointer");
  NutsbDev d = layout(mem, C, P, hist_cap);
  *thprop = d.thprop;
  *hist = d.hist;
  *hist_depth = d.hist_depth;
  return AB_OK;
}

extern "C" int ab_nutsb_advance(void* mem, int C, int P, int hist_cap, int max_depth, double eps, uint64_t seed,
                                uint32_t comp, const double* logp_new, const float* g_new, void* stream) {
  return ab_nutsb_advance_variant(mem, C, P, hist_cap, max_depth, eps, seed, comp, AB_NUTS_REFERENCE, logp_new, g_new,
                                  stream);
}

extern "C" int ab_nutsb_advance_variant(void* mem, int C, int P, int hist_cap, int max_depth, double eps,
                                        uint64_t seed, uint32_t comp, int variant, const double* logp_new,
                                        const float* g_new, void* stream) {
  AB_REQUIRE(variant == AB_NUTS_REFERENCE || variant == AB_NUTS_STANDARD, AB_ERR_ARG,
             "ab_nutsb_advance: unknown variant %d", variant);
  AB_REQUIRE(mem && logp_new && g_new && C > 0 && P > 0, AB_ERR_ARG, "ab_nutsb_advance: bad arguments");
  AB_REQUIRE(max_depth >= 1 && max_depth <= 14, AB_ERR_ARG, "ab_nutsb_advance: max_depth must be 1..14");
  AB_REQUIRE(eps > 0.0 && eps < 1e5, AB_ERR_ARG, "ab_nutsb_advance: bad step size");
  NutsbDev d = layout(mem, C, P, hist_cap);
  d.max_depth = max_depth;
  d.eps = (float)eps;
  d.seed = seed;
  d.comp = comp;
  d.logp_new = logp_new;
  d.g_new = g_new;
  d.standard = variant == AB_NUTS_STANDARD;
  nutsb_advance_kernel<<<C, NB_THREADS, 0, as_stream(stream)>>>(d);
  AB_LAUNCH_CHECK("nutsb_advance_kernel");
  return AB_OK;
}

extern "C" int ab_nutsb_info(void* mem, int C, int P, int hist_cap, double* info, void* stream) {
  AB_REQUIRE(mem && info && C > 0, AB_ERR_ARG, "ab_nutsb_info: bad arguments");
  NutsbDev d = layout(mem, C, P, hist_cap);
  nutsb_info_kernel<<<ceil_div(C, 128), 128, 0, as_stream(stream)>>>(d, info);
  AB_LAUNCH_CHECK("nutsb_info_kernel");
  return AB_OK;
}

extern "C" int ab_nutsb_reset_history(void* mem, int C, int P, int hist_cap, void* stream) {
  AB_REQUIRE(mem && C > 0 && P > 0 && hist_cap >= 0, AB_ERR_ARG, "ab_nutsb_reset_history: bad arguments");
  NutsbDev d = layout(mem, C, P, hist_cap);
  nutsb_reset_history_kernel<<<ceil_div(C, 128), 128, 0, as_stream(stream)>>>(d);
  AB_LAUNCH_CHECK("nutsb_reset_history_kernel");
  return AB_OK;
}

// ---- grouped NUTS: many samplers, one advance launch per round --------------
namespace ab {
namespace {
// Per instance, over its chains: [2i] = the smallest draw count, [2i+1] = 1
// if any chain reported an error.
__global__ void nutsg_min_draws_kernel(const NutsbDev* __restrict__ tab, int* __restrict__ out) {
  __shared__ int mn, bad;
  const NutsbDev& d = tab[blockIdx.x];
  if (threadIdx.x == 0) { mn = 0x7fffffff; bad = 0; }
  __syncthreads();
  int m = 0x7fffffff, e = 0;
  for (int c = threadIdx.x; c < d.C; c += blockDim.x) {
    m = min(m, d.st[c].ndraws);
    e |= d.st[c].error;
  }
  atomicMin(&mn, m);
  if (e) atomicOr(&bad, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = mn;
    out[2 * blockIdx.x + 1] = bad;
  }
}
}  // namespace
}  // namespace ab

struct ab_nutsg {
  int n = 0, C_max = 0, n_active = 0;
  std::vector<ab::NutsbDev> all;   // every instance, in creation order
  ab::NutsbDev* d_all = nullptr;   // the same, on the device (min-draws queries)
  ab::NutsbDev* d_act = nullptr;   // the active instances, compacted
  int* d_n = nullptr;              // number of active instances
};

extern "C" int ab_nutsg_create(int n, const ab_nutsg_inst* insts, ab_nutsg** out) {
  AB_REQUIRE(out && insts && n >= 1 && n <= 65535, AB_ERR_ARG, "ab_nutsg_create: bad arguments");
  *out = nullptr;
  std::unique_ptr<ab_nutsg> g(new ab_nutsg());
  g->n = n;
  for (int i = 0; i < n; ++i) {
    const ab_nutsg_inst& q = insts[i];
    AB_REQUIRE(q.state && q.logp_new && q.g_new && q.C > 0 && q.P > 0 && q.hist_cap >= 0, AB_ERR_ARG,
               "ab_nutsg_create: instance %d: bad arguments", i);
    AB_REQUIRE((reinterpret_cast<uintptr_t>(q.state) & 255) == 0, AB_ERR_ARG,
               "ab_nutsg_create: instance %d: state must be 256-byte aligned", i);
    AB_REQUIRE(q.variant == AB_NUTS_REFERENCE || q.variant == AB_NUTS_STANDARD, AB_ERR_ARG,
               "ab_nutsg_create: instance %d: unknown variant %d", i, q.variant);
    AB_REQUIRE(q.max_depth >= 1 && q.max_depth <= 14, AB_ERR_ARG,
               "ab_nutsg_create: instance %d: max_depth must be 1..14", i);
    AB_REQUIRE(q.eps > 0.0 && q.eps < 1e5, AB_ERR_ARG, "ab_nutsg_create: instance %d: bad step size", i);
    NutsbDev d = layout(q.state, q.C, q.P, q.hist_cap);
    d.max_depth = q.max_depth;
    d.eps = (float)q.eps;
    d.seed = q.seed;
    d.comp = q.comp;
    d.logp_new = q.logp_new;
    d.g_new = q.g_new;
    d.standard = q.variant == AB_NUTS_STANDARD;
    g->all.push_back(d);
    g->C_max = std::max(g->C_max, q.C);
  }
  const size_t tb = sizeof(NutsbDev) * (size_t)n;
  AB_CUDA(cudaMalloc(&g->d_all, tb));
  AB_CUDA(cudaMalloc(&g->d_act, tb));
  AB_CUDA(cudaMalloc(&g->d_n, sizeof(int)));
  AB_CUDA(cudaMemcpy(g->d_all, g->all.data(), tb, cudaMemcpyHostToDevice));
  AB_CUDA(cudaMemcpy(g->d_act, g->all.data(), tb, cudaMemcpyHostToDevice));
  g->n_active = n;
  AB_CUDA(cudaMemcpy(g->d_n, &g->n_active, sizeof(int), cudaMemcpyHostToDevice));
  *out = g.release();
  return AB_OK;
}

extern "C" int ab_nutsg_set_active(ab_nutsg* g, const int* active, void* stream) {
  AB_REQUIRE(g && active, AB_ERR_ARG, "ab_nutsg_set_active: null argument");
  std::vector<NutsbDev> act;
  for (int i = 0; i < g->n; ++i)
    if (active[i]) act.push_back(g->all[i]);
  g->n_active = (int)act.size();
  cudaStream_t st = as_stream(stream);
  if (!act.empty())
    AB_CUDA(cudaMemcpyAsync(g->d_act, act.data(), sizeof(NutsbDev) * act.size(), cudaMemcpyHostToDevice, st));
  AB_CUDA(cudaMemcpyAsync(g->d_n, &g->n_active, sizeof(int), cudaMemcpyHostToDevice, st));
  // the host vectors are pageable: the copies have left them when the calls return
  return AB_OK;
}

extern "C" int ab_nutsg_advance(ab_nutsg* g, void* stream) {
  AB_REQUIRE(g, AB_ERR_ARG, "ab_nutsg_advance: null group");
  nutsg_advance_kernel<<<dim3(g->C_max, g->n), NB_THREADS, 0, as_stream(stream)>>>(g->d_act, g->d_n);
  AB_LAUNCH_CHECK("nutsg_advance_kernel");
  return AB_OK;
}

extern "C" int ab_nutsg_min_draws(ab_nutsg* g, int* out, void* stream) {
  AB_REQUIRE(g && out, AB_ERR_ARG, "ab_nutsg_min_draws: null argument");
  nutsg_min_draws_kernel<<<g->n, 128, 0, as_stream(stream)>>>(g->d_all, out);
  AB_LAUNCH_CHECK("nutsg_min_draws_kernel");
  return AB_OK;
}

extern "C" int ab_nutsg_destroy(ab_nutsg* g) {
  if (!g) return AB_OK;
  cudaFree(g->d_all);
  cudaFree(g->d_act);
  cudaFree(g->d_n);
  delete g;
  return AB_OK;
}
