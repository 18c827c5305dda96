/* Minimal stand-in for the GNU Scientific Library RNG interface, written for this project so that the
 * reference's own CPU sources (which include <gsl/gsl_rng.h>) compile without GSL. Test infrastructure
 * only: nothing in the product links it.
 *
 * Generators (restated from their published descriptions, not from GSL's source):
 *   gsl_rng_ranlxs0  RANLUX subtract-with-borrow, base 2^24, lags (24, 10), luxury p = 218
 *                    (Luescher, Comput. Phys. Commun. 79 (1994) 100; James, ibid. 79 (1994) 111).
 *                    In replay mode (gslshim_set_replay) it serves a caller-supplied stream instead.
 *   gsl_rng_taus     combined Tausworthe generator "taus88" (L'Ecuyer, Math. Comp. 65 (1996) 203).
 * Streams are NOT bit-identical to GSL's: the reference pins no RNG output values, only same-seed
 * reproducibility. */
#ifndef GSLSHIM_RNG_H_
#define GSLSHIM_RNG_H_
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct gsl_rng_type {
  const char *name;
  int kind; /* 0 = ranlux (replayable), 1 = taus88 */
} gsl_rng_type;

typedef struct gsl_rng {
  const gsl_rng_type *type;
  void *state;
} gsl_rng;

extern const gsl_rng_type *gsl_rng_ranlxs0;
extern const gsl_rng_type *gsl_rng_taus;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
double gsl_rng_uniform(const gsl_rng *r);
void gsl_rng_free(gsl_rng *r);
const gsl_rng_type *gsl_rng_env_setup(void);

/* Replay hook: while a replay stream is installed, every gsl_rng_uniform() call on a ranlxs0
 * generator returns the next value of `values` (in call order) instead of a RANLUX draw.
 * Running past the end aborts the process with a message. */
void gslshim_set_replay(const double *values, size_t n);
void gslshim_clear_replay(void);
size_t gslshim_replay_consumed(void);

#ifdef __cplusplus
}
#endif
#endif
