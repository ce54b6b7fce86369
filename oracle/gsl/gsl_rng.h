/*
 * ORACLE (test infrastructure only).  Minimal stand-in for the two GSL
 * headers that the reference runtime includes (cbits/augur_hdr.h:23-24).
 * GSL 2.3 is not available here; the six symbols the reference links are
 * provided by oracle/gsl_shim.c on top of the Philox substream contract.
 */
#ifndef ORACLE_GSL_RNG_H
#define ORACLE_GSL_RNG_H
#include <stddef.h>
#include <stdint.h>

typedef struct gsl_rng_type { const char* name; } gsl_rng_type;
typedef struct gsl_rng { const gsl_rng_type* type; void* state; } gsl_rng;

extern const gsl_rng_type* gsl_rng_default;
void gsl_rng_env_setup(void);
gsl_rng* gsl_rng_alloc(const gsl_rng_type* T);
double gsl_rng_uniform(const gsl_rng* r);

/* Shim extensions: select the Philox substream a generator draws from. */
void orc_shim_set_seed(uint64_t seed);
void orc_shim_seek(const gsl_rng* r, uint32_t elem, uint32_t iter, uint32_t tag);
void orc_shim_seek_elementwise(const gsl_rng* r, uint32_t elem0, uint32_t iter, uint32_t tag);
uint32_t orc_shim_pos(const gsl_rng* r);
#endif
