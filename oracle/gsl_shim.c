/*
 * ORACLE (test infrastructure only).  The six GSL symbols that the reference
 * runtime links (gsl_rng_alloc, gsl_rng_default, gsl_rng_env_setup,
 * gsl_rng_uniform, gsl_ran_gaussian_ziggurat, gsl_ran_exponential; call sites
 * cbits/augur_dist.c:35-40,84,398,459 and cbits/augur_mcmclib.h:75,110,138-141,
 * 513,717), implemented over the Philox substream contract of oracle_rng.h so
 * that the reference's own CPU code consumes the same uniforms as the CUDA
 * library.  GSL itself (2.3, not vendored) is absent: agreement with genuine
 * GSL streams is not claimed.  gsl_ran_gaussian_ziggurat is served by the
 * Box-Muller normal of the contract, not by a ziggurat.
 */
#include <stdlib.h>
#include "gsl/gsl_rng.h"
#include "gsl/gsl_randist.h"
#include "oracle_rng.h"

static const gsl_rng_type orc_philox_type = {"philox4x32_10"};

/* Generator state: a substream cursor, optionally in "element-wise" mode in
 * which draw i is the first draw of substream (elem0 + i, iter, tag); that is
 * how the library addresses per-element draws (momenta) that the reference
 * takes sequentially from one generator. */
typedef struct {
  orc_stream s;
  int elementwise;
  uint32_t next_elem;
} orc_shim_state;
const gsl_rng_type* gsl_rng_default = &orc_philox_type;
static uint64_t orc_seed = 0;

void orc_shim_set_seed(uint64_t seed) { orc_seed = seed; }

void gsl_rng_env_setup(void) {}

gsl_rng* gsl_rng_alloc(const gsl_rng_type* T) {
  gsl_rng* r = (gsl_rng*)malloc(sizeof(gsl_rng));
  orc_shim_state* s = (orc_shim_state*)calloc(1, sizeof(orc_shim_state));
  s->s = orc_make(orc_seed, 0, 0, 0);
  r->type = T;
  r->state = s;
  return r;
}

void orc_shim_seek(const gsl_rng* r, uint32_t elem, uint32_t iter, uint32_t tag) {
  orc_shim_state* s = (orc_shim_state*)r->state;
  s->s = orc_make(orc_seed, elem, iter, tag);
  s->elementwise = 0;
}

void orc_shim_seek_elementwise(const gsl_rng* r, uint32_t elem0, uint32_t iter, uint32_t tag) {
  orc_shim_state* s = (orc_shim_state*)r->state;
  s->s = orc_make(orc_seed, elem0, iter, tag);
  s->elementwise = 1;
  s->next_elem = elem0;
}

static orc_stream* cursor(const gsl_rng* r) {
  orc_shim_state* s = (orc_shim_state*)r->state;
  if (s->elementwise) {
    s->s.elem = s->next_elem++;
    s->s.pos = 0;
  }
  return &s->s;
}

uint32_t orc_shim_pos(const gsl_rng* r) { return ((orc_shim_state*)r->state)->s.pos; }

double gsl_rng_uniform(const gsl_rng* r) { return orc_uniform(cursor(r)); }

double gsl_ran_gaussian_ziggurat(const gsl_rng* r, double sigma) {
  return sigma * orc_normal(cursor(r));
}

double gsl_ran_exponential(const gsl_rng* r, double mu) {
  return -mu * log(orc_uniform(cursor(r)));
}
