// Tridiagonal solve shared by the eigensolver (inverse iteration) and the
// adjoint (resolvent of T).
#pragma once

#include <cuda_runtime.h>

namespace pmx {
namespace dev {

// Solves (T - lam I) x = b in place by Gaussian elimination with partial
// pivoting (the LU has two super-diagonals). u0/u1/u2 are scratch of length n.
__device__ inline void tri_solve(const double* d, const double* e, int n, double lam, double tiny,
                          double* x, double* u0, double* u1, double* u2) {
  double a = d[0] - lam;                  // current pivot-row diagonal
  double c = n > 1 ? e[0] : 0.0;          // current pivot-row first super-diagonal
  double c2 = 0.0;                         // current pivot-row second super-diagonal
  for (int i = 0; i < n - 1; ++i) {
    const double b = e[i];                // sub-diagonal below the pivot
    const double dn = d[i + 1] - lam;     // next row diagonal
    const double en = i + 1 < n - 1 ? e[i + 1] : 0.0;  // next row super-diagonal
    if (fabs(a) >= fabs(b)) {
      if (a == 0.0) a = tiny;
      const double f = b / a;
      u0[i] = a;
      u1[i] = c;
      u2[i] = c2;
      x[i + 1] -= f * x[i];
      a = dn - f * c;
      c = en - f * c2;
      c2 = 0.0;
    } else {
      const double f = a / b;  // swap rows i and i+1
      u0[i] = b;
      u1[i] = dn;
      u2[i] = en;
      const double xi = x[i];
      x[i] = x[i + 1];
      x[i + 1] = xi - f * x[i];
      a = c - f * dn;
      c = c2 - f * en;
      c2 = 0.0;
    }
  }
  if (a == 0.0 || fabs(a) < tiny) a = a < 0 ? -tiny : tiny;
  u0[n - 1] = a;
  x[n - 1] = x[n - 1] / u0[n - 1];
  if (n > 1) x[n - 2] = (x[n - 2] - u1[n - 2] * x[n - 1]) / u0[n - 2];
  for (int i = n - 3; i >= 0; --i) x[i] = (x[i] - u1[i] * x[i + 1] - u2[i] * x[i + 2]) / u0[i];
}

}  // namespace dev
}  // namespace pmx
