/* ORACLE (test infrastructure only): see gsl_rng.h in this folder. */
#ifndef ORACLE_GSL_RANDIST_H
#define ORACLE_GSL_RANDIST_H
#include "gsl_rng.h"
double gsl_ran_gaussian_ziggurat(const gsl_rng* r, double sigma);
double gsl_ran_exponential(const gsl_rng* r, double mu);
#endif
