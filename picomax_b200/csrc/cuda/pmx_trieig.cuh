// Eigenpairs of a real symmetric tridiagonal matrix T (diagonal d, off-diagonal
// e) by one CTA: multisection bisection on Sturm counts for the lowest nval
// eigenvalues, then inverse iteration with modified Gram-Schmidt inside
// eigenvalue clusters for the lowest nvec eigenvectors. Shared by the one-stage
// eigensolver (heev_kernel) and the tridiagonal stage of the two-stage one.
//
// LAPACK's dstebz / dstein (the tridiagonal stages behind Eigen's
// SelfAdjointEigenSolver results in the reference, src/pmx_epm.cpp:232) are
// the published methods restated here: Gershgorin interval, pivmin-guarded
// Sturm counts, bisection to 2 eps |lambda| + 4 pivmin, inverse iteration from
// a pseudo-random start.
#pragma once

#include <cfloat>
#include <cmath>

#include <cuda_runtime.h>

#include "pmx_common.cuh"

namespace pmx {
namespace dev {

constexpr int kTriBisectIters = 200;  // cap; multisection converges in ~15 rounds
constexpr int kTriInvIters = 3;

__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int n, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q < 0.0;
  }
  return c;
}

__device__ __forceinline__ double hash_uniform(unsigned long long a, unsigned long long b) {
  unsigned long long x = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull);
  x ^= x >> 31;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  x ^= x >> 31;
  return ((double)(x >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;  // (-1, 1)
}

// Shared-memory work arrays of the tridiagonal stage.
struct TriWork {
  double* d;     // [n] diagonal
  double* e;     // [n] off-diagonal (e[n-1] unused); negligible entries are zeroed
  double* e2;    // [n] squares of e
  double* red;   // [5+] Gershgorin interval, pivmin, |T|, T finite
  double* lam;   // [nval] eigenvalues
  double* lo;    // [nval] bisection brackets
  double* hi;    // [nval]
  double* xs;    // [blockDim.x] multisection probes
  int* cnt;      // [blockDim.x] their Sturm counts
  int* clus;     // [nvec + 1] cluster starts
  int* misc;     // [4]
};

// Lowest nval eigenvalues of T into lam[] and wout[]. Returns 0, 1 (bisection
// did not converge) or 2 (non-finite eigenvalue). Every thread of the block
// calls it; contains block barriers.
__device__ inline int tri_eigvals(const TriWork& W, int n, int nval, double* __restrict__ wout, int cap = 0) {
  const int iters = cap > 0 ? cap : kTriBisectIters;
  const int tid = threadIdx.x, nthr = blockDim.x;
  double *d = W.d, *e = W.e, *e2 = W.e2, *red = W.red, *lo = W.lo, *hi = W.hi, *xs = W.xs, *lam = W.lam;
  int* cnt = W.cnt;
  // Gershgorin interval, pivmin, and negligible off-diagonals set to zero;
  // a non-finite entry of T (fmin/fmax would skip it) fails the matrix
  if (tid == 0) {
    double glo = d[0], ghi = d[0], emax2 = 0.0, tnorm = 0.0;
    int fin = 1;
    for (int i = 0; i < n; ++i) {
      const double el = i > 0 ? fabs(e[i - 1]) : 0.0, er = i < n - 1 ? fabs(e[i]) : 0.0;
      fin &= (isfinite(d[i]) && isfinite(el) && isfinite(er)) ? 1 : 0;
      glo = fmin(glo, d[i] - el - er);
      ghi = fmax(ghi, d[i] + el + er);
      tnorm = fmax(tnorm, fabs(d[i]) + el + er);
    }
    for (int i = 0; i < n - 1; ++i) {
      if (fabs(e[i]) <= DBL_EPSILON * (fabs(d[i]) + fabs(d[i + 1]))) e[i] = 0.0;
      e2[i] = e[i] * e[i];
      emax2 = fmax(emax2, e2[i]);
    }
    const double pad = 2.0 * DBL_EPSILON * tnorm * n + DBL_MIN;
    red[0] = glo - pad;
    red[1] = ghi + pad;
    red[2] = DBL_MIN * fmax(1.0, emax2);
    red[3] = tnorm;
    red[4] = fin;
  }
  __syncthreads();
  const double pivmin = red[2];
  const bool finite_t = red[4] != 0.0;
  for (int k = tid; k < nval; k += nthr) {
    lo[k] = red[0];
    hi[k] = red[1];
  }
  // multisection: G threads per eigenvalue probe G interior points at once
  const int G = nval > 0 ? max(1, nthr / nval) : 1;
  __syncthreads();
  int converged = 0;
  if (nval > nthr) {
    // more eigenvalues than threads: plain bisection, each thread owns the
    // eigenvalues tid, tid + nthr, ...
    for (int iter = 0; iter < iters; ++iter) {
      int done = 1;
      for (int k = tid; k < nval; k += nthr) {
        double l = lo[k], h = hi[k];
        const double tol = 2.0 * DBL_EPSILON * fmax(fabs(l), fabs(h)) + 4.0 * pivmin;
        if (h - l > tol) {
          const double x = l + 0.5 * (h - l);
          if (sturm_count(d, e2, n, x, pivmin) <= k)
            l = x;
          else
            h = x;
          lo[k] = l;
          hi[k] = h;
          done &= (h - l) <= tol ? 1 : 0;
        }
      }
      done = __syncthreads_and(done);
      if (done) {
        converged = 1;
        break;
      }
    }
  }
  for (int iter = 0; iter < iters && !converged && nval <= nthr; ++iter) {
    const int k = tid / G, g = tid % G;
    if (k < nval) {
      const double l = lo[k], h = hi[k];
      const double x = l + (h - l) * (double)(g + 1) / (double)(G + 1);
      xs[tid] = x;
      cnt[tid] = sturm_count(d, e2, n, x, pivmin);
    }
    __syncthreads();
    int done = 1;
    if (tid < nval) {
      const int kk = tid;
      double l = lo[kk], h = hi[kk];
      const double tol = 2.0 * DBL_EPSILON * fmax(fabs(l), fabs(h)) + 4.0 * pivmin;
      if (h - l > tol) {
        for (int gg = 0; gg < G; ++gg) {
          const int t = kk * G + gg;
          if (cnt[t] <= kk)
            l = fmax(l, xs[t]);
          else
            h = fmin(h, xs[t]);
        }
        lo[kk] = l;
        hi[kk] = h;
        done = (h - l) <= tol;
      }
    }
    done = __syncthreads_and(done);
    if (done) {
      converged = 1;
      break;
    }
  }
  int finite = 1;
  for (int k = tid; k < nval; k += nthr) {
    lam[k] = 0.5 * (lo[k] + hi[k]);
    wout[k] = lam[k];
    finite &= isfinite(lam[k]) ? 1 : 0;
  }
  finite = __syncthreads_and(finite);
  return !(finite && finite_t) ? 2 : (!converged ? 1 : 0);
}

// LU factors of T - lam I with partial pivoting (the U factor has two
// super-diagonals), for repeated solves: per row i the multiplier f (its
// lowest mantissa bit set when rows i and i + 1 were swapped, a change of one
// unit in the last place of f), 1 / pivot, and U's two super-diagonals, each
// array at [i * st] (several threads' arrays interleaved).
__device__ inline void tri_factor(const double* __restrict__ d, const double* __restrict__ e, int n, double lam,
                                  double tiny, double* __restrict__ F, double* __restrict__ I0,
                                  double* __restrict__ U1, double* __restrict__ U2, int st) {
  double a = d[0] - lam;          // current pivot-row diagonal
  double c = n > 1 ? e[0] : 0.0;  // current pivot-row super-diagonal
  for (int i = 0; i < n - 1; ++i) {
    const double b = e[i], dn = d[i + 1] - lam, en = i + 1 < n - 1 ? e[i + 1] : 0.0;
    const size_t o = (size_t)i * st;
    if (fabs(a) >= fabs(b)) {
      if (a == 0.0) a = tiny;
      const double ia = 1.0 / a, f = b * ia;
      F[o] = __longlong_as_double(__double_as_longlong(f) & ~1ll);
      I0[o] = ia;
      U1[o] = c;
      U2[o] = 0.0;
      a = dn - f * c;
      c = en;
    } else {  // swap rows i and i + 1
      const double ib = 1.0 / b, f = a * ib;
      F[o] = __longlong_as_double(__double_as_longlong(f) | 1ll);
      I0[o] = ib;
      U1[o] = dn;
      U2[o] = en;
      a = c - f * dn;
      c = -f * en;
    }
  }
  if (a == 0.0 || fabs(a) < tiny) a = a < 0 ? -tiny : tiny;
  I0[(size_t)(n - 1) * st] = 1.0 / a;
}

// Solves (T - lam I) x = b in place with the factors of tri_factor: x (b on
// entry) at xb[i * xs]. Division-free; the loads run eight rows ahead of the
// recurrences.
__device__ inline void tri_factored_solve(const double* __restrict__ F, const double* __restrict__ I0,
                                          const double* __restrict__ U1, const double* __restrict__ U2, int st, int n,
                                          double* __restrict__ xb, int xs) {
  constexpr int kB = 8;
  double xc = xb[0];
  for (int i0 = 0; i0 < n - 1; i0 += kB) {
    double xv[kB], fv[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u;
      xv[u] = i + 1 < n ? xb[(size_t)(i + 1) * xs] : 0.0;
      fv[u] = i + 1 < n ? F[(size_t)i * st] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u;
      if (i + 1 < n) {
        const bool sw = (__double_as_longlong(fv[u]) & 1ll) != 0;
        const double piv = sw ? xv[u] : xc, oth = sw ? xc : xv[u];
        xb[(size_t)i * xs] = piv;
        xc = oth - fv[u] * piv;
      }
    }
  }
  double x1 = xc * I0[(size_t)(n - 1) * st], x2 = 0.0;  // rows i + 1, i + 2
  xb[(size_t)(n - 1) * xs] = x1;
  for (int i0 = n - 2; i0 >= 0; i0 -= kB) {
    double yv[kB], iv[kB], av[kB], bv[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 - u;
      yv[u] = i >= 0 ? xb[(size_t)i * xs] : 0.0;
      iv[u] = i >= 0 ? I0[(size_t)i * st] : 0.0;
      av[u] = i >= 0 ? U1[(size_t)i * st] : 0.0;
      bv[u] = i >= 0 ? U2[(size_t)i * st] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 - u;
      if (i >= 0) {
        const double xi = (yv[u] - av[u] * x1 - bv[u] * x2) * iv[u];
        xb[(size_t)i * xs] = xi;
        x2 = x1;
        x1 = xi;
      }
    }
  }
}

// Lowest nvec eigenvectors of T (after tri_eigvals) as real vectors in the
// real parts of z[k * n + i] (imaginary parts zero). Clusters of eigenvalues
// closer than 1e-5 |T| are reorthogonalised. One thread per cluster: per
// eigenvalue one LU factorisation of T - lam I (tri_factor, its four arrays
// interleaved by cluster in `scratch`, 4 n nvec doubles at most), then
// kTriInvIters division-free solves from a pseudo-random start. The iterate
// lives in shared memory when xsm is given (n * nvec doubles, interleaved by
// cluster), else in the real parts of its z column. `seed` makes the start
// vectors differ per matrix.
__device__ inline void tri_eigvecs(const TriWork& W, int n, int nvec, double2* __restrict__ z,
                                   double* __restrict__ scratch, unsigned long long seed,
                                   double* __restrict__ xsm = nullptr) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const double* d = W.d;
  const double* e = W.e;
  const double* lam = W.lam;
  const double tnorm = W.red[3];
  if (tid == 0) {
    int nc = 0;
    const double gap = 1e-5 * tnorm;
    for (int k = 0; k < nvec; ++k)
      if (k == 0 || lam[k] - lam[k - 1] > gap) W.clus[nc++] = k;
    W.clus[nc] = nvec;
    W.misc[0] = nc;
  }
  __syncthreads();
  const int ncl = W.misc[0];
  const double tiny = DBL_EPSILON * fmax(tnorm, DBL_MIN);
  for (int cl = tid; cl < ncl; cl += nthr) {
    double* F = scratch + cl;
    double* I0 = F + (size_t)n * ncl;
    double* U1 = I0 + (size_t)n * ncl;
    double* U2 = U1 + (size_t)n * ncl;
    for (int k = W.clus[cl]; k < W.clus[cl + 1]; ++k) {
      double* xb = xsm ? xsm + cl : reinterpret_cast<double*>(z + (size_t)k * n);
      const int xs = xsm ? ncl : 2;
      auto X = [&](int i) -> double& { return xb[(size_t)i * xs]; };
      tri_factor(d, e, n, lam[k], tiny, F, I0, U1, U2, ncl);
      for (int i = 0; i < n; ++i) X(i) = hash_uniform((seed << 20) + k, i);
      for (int iter = 0; iter < kTriInvIters; ++iter) {
        tri_factored_solve(F, I0, U1, U2, ncl, n, xb, xs);
        for (int kp = W.clus[cl]; kp < k; ++kp) {
          const double2* zp = z + (size_t)kp * n;
          double s = 0.0;
          for (int i = 0; i < n; ++i) s += zp[i].x * X(i);
          for (int i = 0; i < n; ++i) X(i) -= s * zp[i].x;
        }
        double mx = 0.0;
        for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(X(i)));
        if (!(mx > 0.0) || !isfinite(mx)) mx = 1.0;
        const double imx = 1.0 / mx;
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
          const double v = X(i) * imx;
          X(i) = v;
          s += v * v;
        }
        s = 1.0 / sqrt(s);
        for (int i = 0; i < n; ++i) X(i) *= s;
      }
      double2* zk = z + (size_t)k * n;
      for (int i = 0; i < n; ++i) zk[i] = make_double2(X(i), 0.0);
    }
  }
  __syncthreads();
}

}  // namespace dev
}  // namespace pmx
