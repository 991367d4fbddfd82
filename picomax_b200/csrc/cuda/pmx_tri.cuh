// Tridiagonal solve shared by the eigensolver (inverse iteration) and the
// adjoint (resolvent of T).
#pragma once

#include <cuda_runtime.h>

namespace pmx {
namespace dev {

// Solves (T - lam I) x = b in place by Gaussian elimination with partial
// pivoting (the LU has two super-diagonals). u0/u1/u2 are scratch of length n;
// element i of x, u0, u1, u2 is at [i * st] (st > 1: the arrays of several
// threads interleaved, so that a warp's accesses to row i coalesce). The
// current row of the elimination and the last two solution values of the
// back substitution stay in registers (no reload of a value just stored).
__device__ inline void tri_solve(const double* __restrict__ d, const double* __restrict__ e, int n, double lam,
                                 double tiny, double* __restrict__ x, double* __restrict__ u0,
                                 double* __restrict__ u1, double* __restrict__ u2, int st = 1) {
  auto X = [&](int i) -> double& { return x[(size_t)i * st]; };
  auto U0 = [&](int i) -> double& { return u0[(size_t)i * st]; };
  auto U1 = [&](int i) -> double& { return u1[(size_t)i * st]; };
  auto U2 = [&](int i) -> double& { return u2[(size_t)i * st]; };
  double a = d[0] - lam;                  // current pivot-row diagonal
  double c = n > 1 ? e[0] : 0.0;          // current pivot-row first super-diagonal
  double c2 = 0.0;                         // current pivot-row second super-diagonal
  double xc = X(0);                        // current pivot-row right-hand side
  for (int i = 0; i < n - 1; ++i) {
    const double xn = X(i + 1);           // right-hand side of row i + 1
    const double b = e[i];                // sub-diagonal below the pivot
    const double dn = d[i + 1] - lam;     // next row diagonal
    const double en = i + 1 < n - 1 ? e[i + 1] : 0.0;  // next row super-diagonal
    if (fabs(a) >= fabs(b)) {
      if (a == 0.0) a = tiny;
      const double f = b / a;
      U0(i) = a;
      U1(i) = c;
      U2(i) = c2;
      X(i) = xc;
      xc = xn - f * xc;
      a = dn - f * c;
      c = en - f * c2;
      c2 = 0.0;
    } else {
      const double f = a / b;  // swap rows i and i+1
      U0(i) = b;
      U1(i) = dn;
      U2(i) = en;
      X(i) = xn;
      xc = xc - f * xn;
      a = c - f * dn;
      c = c2 - f * en;
      c2 = 0.0;
    }
  }
  if (a == 0.0 || fabs(a) < tiny) a = a < 0 ? -tiny : tiny;
  U0(n - 1) = a;
  double x1 = xc / a, x2 = 0.0;  // rows i + 1 and i + 2 of the back substitution
  X(n - 1) = x1;
  if (n > 1) {
    x2 = x1;
    x1 = (X(n - 2) - U1(n - 2) * x2) / U0(n - 2);
    X(n - 2) = x1;
  }
  for (int i = n - 3; i >= 0; --i) {
    const double xi = (X(i) - U1(i) * x1 - U2(i) * x2) / U0(i);
    X(i) = xi;
    x2 = x1;
    x1 = xi;
  }
}

}  // namespace dev
}  // namespace pmx
