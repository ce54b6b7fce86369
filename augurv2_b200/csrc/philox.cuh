// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), shared by every
// kernel of this library.
//
// The reference draws from one sequential GSL stream on the CPU
// (cbits/augur_dist.c:33-47, :396-402, :457-463) and from per-index curand
// states on the GPU (compiler/augur/src/CudaC/CgCuda.hs:116-122).  Here every
// draw is addressed instead: a *substream* is the 4-word counter
// (draw, element, iteration, tag) under a 64-bit key (the seed), and a
// substream is consumed sequentially over its first word.  Each uniform and
// each normal consumes exactly one Philox block, so a substream position is
// the number of draws made from it.  The same addressing is used by the CPU
// oracle, which is how both sides are "fed the same uniforms".
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define AB_HD __host__ __device__ __forceinline__
#else
#define AB_HD static inline
#endif

namespace ab {

struct Philox4 {
  uint32_t x[4];
};

AB_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

// One Philox4x32-10 block: 10 rounds of the (M0, M1) multiply-xor bijection,
// with the Weyl key schedule (W0, W1) between rounds.
AB_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                            uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = mulhi32(M0, c0), lo0 = M0 * c0;
    uint32_t hi1 = mulhi32(M1, c2), lo1 = M1 * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += W0; k1 += W1;
  }
  Philox4 out;
  out.x[0] = c0; out.x[1] = c1; out.x[2] = c2; out.x[3] = c3;
  return out;
}

// 52 random bits -> double in the open interval (0, 1).  (m + 0.5) * 2^-52
// is exact in binary64, so host and device produce identical bits.
AB_HD double bits_to_unit(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)(a & 0xFFFFFu) << 32) | (uint64_t)b;
  return ((double)m + 0.5) * 2.220446049250313080847263336181640625e-16;
}

// Tags of the fourth counter word (low 8 bits); the upper 24 bits carry the
// chain / instance index for batched samplers.
enum Tag : uint32_t {
  TAG_Z = 1,          // discrete Gibbs: one uniform per latent
  TAG_THETA = 2,      // Dirichlet conjugate draw, first block (LDA theta)
  TAG_PHI = 3,        // Dirichlet conjugate draw, second block (LDA phi)
  TAG_MOM = 4,        // HMC / NUTS momentum
  TAG_HMC = 5,        // HMC jitter + accept (host-rng role)
  TAG_NUTS = 6,       // NUTS slice + direction + subtree choices
  TAG_PI = 7,         // GMM mixture weights
  TAG_MU = 8,         // GMM means
  TAG_COV = 9,        // GMM covariances
  TAG_ESLICE = 10,    // elliptical slice
  TAG_MWG = 11,       // Metropolis-within-Gibbs
  TAG_INIT = 12,      // initial points
  TAG_DATA = 13,      // synthetic data
  TAG_RSLICE = 14,    // reflective slice: the slice level's exponential
  TAG_CONJ = 15,      // scalar conjugate updates
};

// A sequential cursor over one substream.
struct Stream {
  uint32_t k0, k1;       // key (seed)
  uint32_t elem, iter, tag;
  uint32_t pos;          // draws consumed so far

  AB_HD Philox4 next_block() {
    Philox4 r = philox4x32_10(pos, elem, iter, tag, k0, k1);
    ++pos;
    return r;
  }
  AB_HD double uniform() {
    Philox4 r = next_block();
    return bits_to_unit(r.x[0], r.x[1]);
  }
  // Standard normal by the Box-Muller transform (Box & Muller 1958) on the
  // two uniforms of one block; only the cosine branch is used so that every
  // normal costs exactly one block.
  AB_HD double normal() {
    Philox4 r = next_block();
    double u1 = bits_to_unit(r.x[0], r.x[1]);
    double u2 = bits_to_unit(r.x[2], r.x[3]);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925286766559 * u2);
  }
};

AB_HD Stream make_stream(uint64_t seed, uint32_t elem, uint32_t iter, uint32_t tag) {
  Stream s;
  s.k0 = (uint32_t)seed;
  s.k1 = (uint32_t)(seed >> 32);
  s.elem = elem; s.iter = iter; s.tag = tag; s.pos = 0;
  return s;
}

}  // namespace ab
