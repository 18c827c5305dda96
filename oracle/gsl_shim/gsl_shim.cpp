// Stand-in implementation of the GSL calls made by the reference's CPU sources (see gsl/*.h here).
// Test infrastructure only: it lets the reference's own code be compiled as the oracle and the timed CPU
// baseline. Every algorithm below is restated from its published description (cited at each function).
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_eigen.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_rng.h"

static const gsl_rng_type k_ranlux = {"ranlxs0", 0};
static const gsl_rng_type k_taus = {"taus", 1};
const gsl_rng_type *gsl_rng_ranlxs0 = &k_ranlux;
const gsl_rng_type *gsl_rng_taus = &k_taus;

// ---- RANLUX: subtract-with-borrow x_n = x_{n-10} - x_{n-24} - c (mod 2^24), keeping 24 of every 218 values
// (Marsaglia & Zaman 1991 for the SWB recurrence; Luescher 1994 for the decimation; James 1994 for the
// 24-bit formulation and the seeding LCG of L'Ecuyer 1988).
struct Ranlux {
  int32_t x[24];
  int i, j;   // lag pointers (i: lag 24, j: lag 10)
  int carry;
  int kept;   // values delivered since the last skip
};
static const int kLuxury = 218;

static void ranlux_seed(Ranlux *s, unsigned long seed) {
  long j = (long)(seed % 2147483563UL);
  if (j == 0) j = 314159265;
  for (int n = 0; n < 24; n++) {
    long k = j / 53668;
    j = 40014 * (j - k * 53668) - k * 12211;
    if (j < 0) j += 2147483563;
    s->x[n] = (int32_t)(j % 16777216);
  }
  s->carry = s->x[23] == 0 ? 1 : 0;
  s->i = 23;
  s->j = 9;
  s->kept = 0;
}

static inline int32_t ranlux_step(Ranlux *s) {
  int32_t v = s->x[s->j] - s->x[s->i] - s->carry;
  if (v < 0) {
    v += 16777216;
    s->carry = 1;
  } else {
    s->carry = 0;
  }
  s->x[s->i] = v;
  s->i = s->i == 0 ? 23 : s->i - 1;
  s->j = s->j == 0 ? 23 : s->j - 1;
  return v;
}

static double ranlux_uniform(Ranlux *s) {
  int32_t v = ranlux_step(s);
  if (++s->kept == 24) {
    for (int n = 0; n < kLuxury - 24; n++) ranlux_step(s);
    s->kept = 0;
  }
  return v * (1.0 / 16777216.0);
}

// ---- taus88 (L'Ecuyer 1996, "Maximally equidistributed combined Tausworthe generators").
struct Taus {
  uint32_t s1, s2, s3;
};
static void taus_seed(Taus *t, unsigned long seed) {
  uint32_t v = (uint32_t)(seed ? seed : 1);
  v = 69069u * v;
  t->s1 = v < 2u ? v + 2u : v;
  v = 69069u * v;
  t->s2 = v < 8u ? v + 8u : v;
  v = 69069u * v;
  t->s3 = v < 16u ? v + 16u : v;
  for (int n = 0; n < 6; n++) {  // warm up
    uint32_t b = (((t->s1 << 13) ^ t->s1) >> 19);
    t->s1 = (((t->s1 & 4294967294u) << 12) ^ b);
  }
}
static double taus_uniform(Taus *t) {
  uint32_t b;
  b = (((t->s1 << 13) ^ t->s1) >> 19);
  t->s1 = (((t->s1 & 4294967294u) << 12) ^ b);
  b = (((t->s2 << 2) ^ t->s2) >> 25);
  t->s2 = (((t->s2 & 4294967288u) << 4) ^ b);
  b = (((t->s3 << 3) ^ t->s3) >> 11);
  t->s3 = (((t->s3 & 4294967280u) << 17) ^ b);
  return (t->s1 ^ t->s2 ^ t->s3) * (1.0 / 4294967296.0);
}

// ---- replay stream
static const double *g_replay = 0;
static size_t g_replay_n = 0, g_replay_pos = 0;

extern "C" void gslshim_set_replay(const double *values, size_t n) {
  g_replay = values;
  g_replay_n = n;
  g_replay_pos = 0;
}
extern "C" void gslshim_clear_replay(void) {
  g_replay = 0;
  g_replay_n = g_replay_pos = 0;
}
extern "C" size_t gslshim_replay_consumed(void) { return g_replay_pos; }

extern "C" gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) {
  gsl_rng *r = (gsl_rng *)malloc(sizeof(gsl_rng));
  r->type = T;
  if (T->kind == 0) {
    r->state = calloc(1, sizeof(Ranlux));
    ranlux_seed((Ranlux *)r->state, 0);
  } else {
    r->state = calloc(1, sizeof(Taus));
    taus_seed((Taus *)r->state, 0);
  }
  return r;
}

extern "C" void gsl_rng_set(const gsl_rng *r, unsigned long int seed) {
  if (r->type->kind == 0)
    ranlux_seed((Ranlux *)r->state, seed);
  else
    taus_seed((Taus *)r->state, seed);
}

extern "C" double gsl_rng_uniform(const gsl_rng *r) {
  if (r->type->kind == 0) {
    if (g_replay) {
      if (g_replay_pos >= g_replay_n) {
        fprintf(stderr, "gsl_shim: replay stream exhausted after %zu values\n", g_replay_n);
        abort();
      }
      return g_replay[g_replay_pos++];
    }
    return ranlux_uniform((Ranlux *)r->state);
  }
  return taus_uniform((Taus *)r->state);
}

extern "C" void gsl_rng_free(gsl_rng *r) {
  if (!r) return;
  free(r->state);
  free(r);
}

extern "C" const gsl_rng_type *gsl_rng_env_setup(void) { return gsl_rng_ranlxs0; }

// Marsaglia (1972): (u, v) uniform in the unit disc, s = u^2 + v^2; the point
// (2u sqrt(1-s), 2v sqrt(1-s), 1-2s) is uniform on the sphere.
extern "C" void gsl_ran_dir_3d(const gsl_rng *r, double *x, double *y, double *z) {
  double u, v, s;
  do {
    u = 2.0 * gsl_rng_uniform(r) - 1.0;
    v = 2.0 * gsl_rng_uniform(r) - 1.0;
    s = u * u + v * v;
  } while (s >= 1.0 || s == 0.0);
  double a = 2.0 * sqrt(1.0 - s);
  *x = u * a;
  *y = v * a;
  *z = 1.0 - 2.0 * s;
}

// ---- matrices, vectors, symmetric eigensolver
extern "C" gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) {
  gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
  m->size1 = n1;
  m->size2 = n2;
  m->data = (double *)calloc(n1 * n2, sizeof(double));
  return m;
}
extern "C" void gsl_matrix_free(gsl_matrix *m) {
  if (!m) return;
  free(m->data);
  free(m);
}
extern "C" void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { m->data[i * m->size2 + j] = x; }
extern "C" double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->size2 + j]; }
extern "C" gsl_vector *gsl_vector_alloc(size_t n) {
  gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
  v->size = n;
  v->data = (double *)calloc(n, sizeof(double));
  return v;
}
extern "C" void gsl_vector_free(gsl_vector *v) {
  if (!v) return;
  free(v->data);
  free(v);
}
extern "C" double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i]; }

extern "C" gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n) {
  gsl_eigen_symmv_workspace *w = (gsl_eigen_symmv_workspace *)malloc(sizeof(*w));
  w->size = n;
  return w;
}
extern "C" void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { free(w); }

// Cyclic Jacobi: annihilate each off-diagonal element in turn with a plane rotation until the
// off-diagonal norm is negligible (Golub & Van Loan, Algorithm 8.5.3).
extern "C" int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w) {
  const size_t n = A->size1;
  double *a = A->data, *v = evec->data;
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j < n; j++) v[i * n + j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, diag = 0;
    for (size_t i = 0; i < n; i++) {
      diag += a[i * n + i] * a[i * n + i];
      for (size_t j = i + 1; j < n; j++) off += a[i * n + j] * a[i * n + j];
    }
    if (off <= 1e-34 * diag || off == 0) break;
    for (size_t p = 0; p < n; p++) {
      for (size_t q = p + 1; q < n; q++) {
        double apq = a[p * n + q];
        if (apq == 0) continue;
        double theta = (a[q * n + q] - a[p * n + p]) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        double c = 1 / sqrt(t * t + 1), s = t * c;
        for (size_t k = 0; k < n; k++) {  // A <- A J
          double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (size_t k = 0; k < n; k++) {  // A <- J^T A
          double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (size_t k = 0; k < n; k++) {  // V <- V J
          double vkp = v[k * n + p], vkq = v[k * n + q];
          v[k * n + p] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
    }
  }
  for (size_t i = 0; i < n; i++) eval->data[i] = a[i * n + i];
  (void)w;
  return 0;
}

extern "C" int gsl_eigen_symmv_sort(gsl_vector *eval, gsl_matrix *evec, gsl_eigen_sort_t sort_type) {
  const size_t n = eval->size;
  for (size_t i = 0; i < n; i++) {
    size_t best = i;
    for (size_t j = i + 1; j < n; j++) {
      double a = eval->data[j], b = eval->data[best];
      int better = 0;
      switch (sort_type) {
        case GSL_EIGEN_SORT_VAL_ASC: better = a < b; break;
        case GSL_EIGEN_SORT_VAL_DESC: better = a > b; break;
        case GSL_EIGEN_SORT_ABS_ASC: better = fabs(a) < fabs(b); break;
        case GSL_EIGEN_SORT_ABS_DESC: better = fabs(a) > fabs(b); break;
      }
      if (better) best = j;
    }
    if (best != i) {
      double t = eval->data[i];
      eval->data[i] = eval->data[best];
      eval->data[best] = t;
      for (size_t k = 0; k < n; k++) {
        double u = evec->data[k * n + i];
        evec->data[k * n + i] = evec->data[k * n + best];
        evec->data[k * n + best] = u;
      }
    }
  }
  return 0;
}
