#ifndef GG_SHIM_GSL_RANDIST_H
#define GG_SHIM_GSL_RANDIST_H
#include "gsl_rng.h"
double gsl_ran_gaussian(gsl_rng *r, double sigma);
double gsl_ran_ugaussian(gsl_rng *r);
unsigned int gsl_ran_poisson(gsl_rng *r, double mu);
#endif
