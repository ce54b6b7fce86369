/*
 * ORACLE (test infrastructure only).  Stand-in for the per-model header that
 * the reference compiler generates (written by pyaugur/pyaugur/augurlib.py:
 * 318-332, included by cbits/augur_mcmclib.h:26).  It declares the model
 * state records that the restated generated functions in ref_models.c pass
 * to the reference's MCMC kernels.
 */
#ifndef AUGUR_IFACE_H
#define AUGUR_IFACE_H
#include <augur_vecop.h>
#include <augur_dist.h>

typedef struct AugurMod {
  double* par;         /* HLR: [theta[0..D-1], b, v] */
  AugurVec_t* mu;      /* GMM means (ESlice / MWG), [K] rows of d */
} AugurMod_t;

typedef struct AugurAux {
  augur_rng* rng;
  void* model;         /* model-specific data record (ref_models.c) */
} AugurAux_t;

#endif
