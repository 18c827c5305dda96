/* Stand-in for <gsl/gsl_randist.h> (test infrastructure): gsl_ran_dir_3d draws an isotropic unit
 * vector by Marsaglia's method (Ann. Math. Stat. 43 (1972) 645). */
#ifndef GSLSHIM_RANDIST_H_
#define GSLSHIM_RANDIST_H_
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
void gsl_ran_dir_3d(const gsl_rng *r, double *x, double *y, double *z);
#ifdef __cplusplus
}
#endif
#endif
