/* Stand-in for the small part of <gsl/gsl_eigen.h> the reference uses (test infrastructure):
 * dense matrices/vectors and the symmetric eigensolver, implemented as cyclic Jacobi rotations in
 * FP64 (Golub & Van Loan, Matrix Computations, sec. 8.5). */
#ifndef GSLSHIM_EIGEN_H_
#define GSLSHIM_EIGEN_H_
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct gsl_matrix {
  size_t size1, size2;
  double *data; /* row-major */
} gsl_matrix;

typedef struct gsl_vector {
  size_t size;
  double *data;
} gsl_vector;

typedef struct gsl_eigen_symmv_workspace {
  size_t size;
} gsl_eigen_symmv_workspace;

typedef enum { GSL_EIGEN_SORT_VAL_ASC, GSL_EIGEN_SORT_VAL_DESC, GSL_EIGEN_SORT_ABS_ASC, GSL_EIGEN_SORT_ABS_DESC } gsl_eigen_sort_t;

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);

gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
/* Eigenvalues into eval, eigenvectors as the columns of evec. A is used as scratch. */
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv_sort(gsl_vector *eval, gsl_matrix *evec, gsl_eigen_sort_t sort_type);

#ifdef __cplusplus
}
#endif
#endif
