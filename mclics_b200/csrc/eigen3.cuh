// Largest eigenpair of a symmetric 3x3 matrix in FP64 by cyclic Jacobi rotations (Golub & Van Loan,
// "Matrix Computations", Algorithm 8.5.3). Replaces gsl_eigen_symmv + sort (src/parameter_order.cpp:19-37),
// which the reference uses to get S (largest eigenvalue of Q) and the director (its eigenvector).
#pragma once
#include <math.h>

namespace mcl {

__host__ __device__ inline double largest_eigen3(const double q6[6], double vec[3]) {
  double a[3][3] = {{q6[0], q6[1], q6[2]}, {q6[1], q6[3], q6[4]}, {q6[2], q6[4], q6[5]}};
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 50; sweep++) {
    double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off == 0 || off <= 1e-34 * dg) break;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        double apq = a[p][q];
        if (apq == 0) continue;
        double theta = (a[q][q] - a[p][p]) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        double c = 1 / sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 3; k++) {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; k++) {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; k++) {
          double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int best = 0;
  if (a[1][1] > a[best][best]) best = 1;
  if (a[2][2] > a[best][best]) best = 2;
  vec[0] = v[0][best];
  vec[1] = v[1][best];
  vec[2] = v[2][best];
  return a[best][best];
}

}  // namespace mcl
