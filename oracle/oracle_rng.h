/*
 * ORACLE (test infrastructure only).  Plain-C restatement of the random
 * number contract shared with the CUDA library: Philox4x32-10 (Salmon et al.,
 * SC'11) addressed as substreams (draw, element, iteration, tag) under a
 * 64-bit key.  Written independently of the library's CUDA header so that the
 * known-answer vectors pin both.  Only tests, the smoke check and the CPU
 * baseline leg of the benchmark may use this file.
 */
#ifndef ORACLE_RNG_H
#define ORACLE_RNG_H
#include <math.h>
#include <stdint.h>

typedef struct {
  uint32_t k0, k1, elem, iter, tag, pos;
} orc_stream;

static inline void orc_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline orc_stream orc_make(uint64_t seed, uint32_t elem, uint32_t iter, uint32_t tag) {
  orc_stream s;
  s.k0 = (uint32_t)seed; s.k1 = (uint32_t)(seed >> 32);
  s.elem = elem; s.iter = iter; s.tag = tag; s.pos = 0;
  return s;
}

static inline void orc_block(orc_stream* s, uint32_t out[4]) {
  uint32_t ctr[4] = {s->pos, s->elem, s->iter, s->tag};
  orc_philox(ctr, s->k0, s->k1, out);
  s->pos++;
}

/* (m + 1/2) 2^-52 with m the low 52 bits of (a, b): exact, in (0, 1). */
static inline double orc_unit(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)(a & 0xFFFFFu) << 32) | (uint64_t)b;
  return ((double)m + 0.5) * 2.220446049250313080847263336181640625e-16;
}

static inline double orc_uniform(orc_stream* s) {
  uint32_t o[4];
  orc_block(s, o);
  return orc_unit(o[0], o[1]);
}

/* Box-Muller (cosine branch), one block per normal. */
static inline double orc_normal(orc_stream* s) {
  uint32_t o[4];
  orc_block(s, o);
  double u1 = orc_unit(o[0], o[1]);
  double u2 = orc_unit(o[2], o[3]);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925286766559 * u2);
}

enum {
  ORC_TAG_Z = 1, ORC_TAG_THETA = 2, ORC_TAG_PHI = 3, ORC_TAG_MOM = 4,
  ORC_TAG_HMC = 5, ORC_TAG_NUTS = 6, ORC_TAG_PI = 7, ORC_TAG_MU = 8,
  ORC_TAG_COV = 9, ORC_TAG_ESLICE = 10, ORC_TAG_MWG = 11, ORC_TAG_INIT = 12,
  ORC_TAG_DATA = 13, ORC_TAG_RSLICE = 14, ORC_TAG_CONJ = 15
};

#endif
