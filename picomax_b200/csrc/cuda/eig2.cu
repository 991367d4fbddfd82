// Two-stage batched FP64 Hermitian eigensolver: dense -> band -> tridiagonal.
//
// Replaces Eigen::SelfAdjointEigenSolver (src/pmx_epm.cpp:232, :402,
// src/pmx_chi.cpp:388, :476) for the sizes whose matrix does not fit in
// shared memory. The one-stage reduction (epm.cu) streams the whole trailing
// block through L2/HBM once per column; here the Householder reduction is
// split the way blocked LAPACK/PLASMA solvers split it (Bischof, Lang, Sun,
// "A framework for symmetric band reduction", ACM TOMS 26 (2000); Haidar,
// Ltaief, Dongarra, SC'11), each stage B200-shaped:
//
//  1. sb_kernel (one CTA per matrix): panels of 16 columns. A panel is
//     QR-factorised in shared memory (Householder, compact WY T factor), then
//     the trailing block is updated two-sidedly with two passes of 16 x 16
//     complex tiles on the FP64 tensor cores (mma.sync m8n8k4 .f64):
//       Y = A V          (all tiles, the upper ones read as conj-transposes)
//       X = Y T - 1/2 V (T^H V^H Y T)
//       A -= V X^H + X V^H   (lower tiles and the diagonal tiles in full)
//     Each pass reads (and the second writes) the trailing block once per
//     panel instead of once per column. The panel's reflectors stay in place
//     below the band (LAPACK layout); T goes into the free upper tile.
//  2. sbtrd_kernel (one CTA per matrix): the band (16 sub-diagonals plus 16
//     for the bulge) lives in shared memory; sweeps chase their bulges down
//     the band, each sweep three time steps behind the previous one so that
//     the tasks of one time step touch disjoint rows (one warp per task, one
//     barrier per time step). Reflectors go to global memory.
//  3. tri_eig_kernel: bisection and inverse iteration on the tridiagonal
//     matrix (pmx_trieig.cuh), one CTA per matrix with small shared memory,
//     so that many matrices share an SM.
//  4. eig2_back_kernel: eigenvectors of T -> of the band (the bulge-chasing
//     reflectors of one sweep act on disjoint rows: all applied at once, the
//     sweeps in reverse) -> of H (the panels' compact WY factors in reverse).
//
// The matrix dimension is padded to ld = a multiple of 16 with zero rows and
// columns: every reflector then has zero components in the padding, so T is
// block diagonal with the n x n block of the unpadded problem (e[n-1] = 0
// exactly) and the eigenvectors are exactly zero in the padding.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "pmx_common.cuh"
#include "pmx_device.hpp"
#include "pmx_trieig.cuh"

namespace pmx {
namespace dev {

namespace {

constexpr int kNB = 16;        // panel width = band width
constexpr int kThr = 256;      // threads per CTA of every stage
constexpr int kNW = kThr / 32;
constexpr int kLag = 3;        // time steps between consecutive sweeps
constexpr int kMaxLd = 416;    // largest padded dimension (shared memory of both stages)
constexpr int kVecBlock = 32;  // eigenvectors per back-transform CTA

// element (r, c) of an m x 16 complex panel in shared memory: rows of 16,
// columns XOR-swizzled by the row so that the tensor-core fragment loads of
// 8 rows x 4 columns and of 4 rows x 8 columns are free of bank conflicts
__device__ __forceinline__ int pidx(int r, int c) { return r * kNB + (c ^ (r & 7)); }

// D += A B for one 8x8 (A 8x4 row-major, B 4x8 column-major) FP64 MMA.
// Fragments: a = A[lane/4][lane%4], b = B[lane%4][lane/4],
// d0/d1 = D[lane/4][2 (lane%4) + 0/1].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// acc (re/im 8x8 block) += a * b in complex arithmetic, four real MMAs
__device__ __forceinline__ void cmma(double (&cr)[2], double (&ci)[2], double2 a, double2 b) {
  dmma(cr[0], cr[1], a.x, b.x);
  dmma(cr[0], cr[1], -a.y, b.y);
  dmma(ci[0], ci[1], a.x, b.y);
  dmma(ci[0], ci[1], a.y, b.x);
}

// acc -= a * conj(b') where the B fragment element is b'(row k, col j) taken
// from a matrix stored as X[j][k] (so the product is V X^H)
__device__ __forceinline__ void cmma_sub_herm(double (&cr)[2], double (&ci)[2], double2 a, double2 x) {
  dmma(cr[0], cr[1], -a.x, x.x);
  dmma(cr[0], cr[1], -a.y, x.y);
  dmma(ci[0], ci[1], a.x, x.y);
  dmma(ci[0], ci[1], -a.y, x.x);
}

// sum over the first `w` lanes' groups: xor reductions within 16 lanes
__device__ __forceinline__ double sum16(double v) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Householder reflector in the zlarfg convention: H^H (alpha; x) = (beta; 0),
// H = I - tau v v^H, v[0] = 1, beta real. From alpha and |x|^2 gives tau, beta
// and the scale 1 / (alpha - beta) of x.
struct Refl {
  double2 tau;
  double beta;
  double2 scal;
};
__device__ __forceinline__ Refl make_refl(double2 alpha, double xn) {
  Refl r;
  if (xn == 0.0 && alpha.y == 0.0) {
    r.tau = make_double2(0, 0);
    r.beta = alpha.x;
    r.scal = make_double2(1, 0);
  } else {
    // two independent divisions: 1 / beta and 1 / |alpha - beta|^2
    r.beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn), alpha.x);
    const double2 den = make_double2(alpha.x - r.beta, alpha.y);
    const double ib = 1.0 / r.beta, idd = 1.0 / (den.x * den.x + den.y * den.y);
    r.tau = make_double2(1.0 - alpha.x * ib, -alpha.y * ib);
    r.scal = make_double2(den.x * idd, -den.y * idd);
  }
  return r;
}

// number of bulge-chasing tasks (= reflectors) of sweep s of an ld x ld band
__host__ __device__ __forceinline__ int sweep_steps(int ld, int s) { return (ld - 1 - s + kNB - 1) / kNB; }
// sum_{m=1}^{M} ceil(m / 16)
__host__ __device__ __forceinline__ long long ceil_sum(long long M) {
  const long long q = M / kNB, r = M % kNB;
  return kNB * q * (q + 1) / 2 + r * (q + 1);
}
// index of the first reflector of sweep s
__host__ __device__ __forceinline__ long long sweep_first(int ld, int s) { return ceil_sum(ld - 1) - ceil_sum(ld - 1 - s); }

// ------------------------------------------------------------------ stage 1
struct SbSmem {
  double2* V;     // [mmax * 16] panel / reflectors V (explicit unit lower trapezoid)
  double2* Y;     // [mmax * 16] Y = A V, then X
  double2* T;     // [16 * 17]
  double2* M;     // [16 * 17] V^H Y (the panel QR's T dots before that)
  double2* P;     // [16 * 17] T^H M
  double2* taus;  // [16]
  // panel QR work arrays, inside Y (free until Y = A V is formed)
  double2* part;  // [2][16][16] partial sums of the panel QR
  double2* rowj;  // [2][16] the current row of the panel QR
  double2* pvw;   // [8][2][MR] per-warp pivot buffers of the panel QR
};

// register rows per thread of the panel QR for a padded dimension ld
inline int sb_rows(int ld) { return ld <= 160 ? 9 : (ld <= 288 ? 17 : 25); }

__host__ __device__ inline size_t sb_smem_bytes(int ld) {
  const int mmax = ld - kNB;
  return sizeof(double2) * ((size_t)2 * mmax * kNB + 3 * kNB * 17 + kNB);
}

// Householder QR of the m x 16 panel (rows r0.. of columns c0..c0+15 of A)
// and its compact WY factor T; leaves R and the reflectors in A (LAPACK
// layout: R on and above the diagonal, v below it) and the explicit V (unit
// diagonal, zeros above) in shared memory. Thread (column c = tid % 16,
// row group g = tid / 16) holds rows g, g + 16, ... of column c in registers.
// Per column j one CTA-wide reduction of one value per thread: for c > j the
// dot conj(a_j)^T a_c (which gives v^H a_c once the reflector's scale is
// known), for c = j the norm |x|^2, for c < j the dot v_c^H a_j (which gives
// the T column, zlarft). The pivot column reaches the threads of a row group
// through the warp's own shared-memory buffer (the group's 16 threads share
// a warp). red/rowj: [2][16][16] / [2][16]; pvw [8][2][MR]; dsm [16][16];
// tsm [16]; T [16][17].
template <int MR>
__device__ void panel_qr(double2* __restrict__ A, int ld, int c0, int r0, int m, double2* V, double2* T,
                         double2* red, double2* rowj, double2* pvw, double2* dsm, double2* tsm) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int c = tid & 15, g = tid >> 4;
  double2* pv = pvw + (size_t)wid * 2 * MR + (g & 1) * MR;  // this group's pivot buffer
  double2 col[MR];
#pragma unroll
  for (int t = 0; t < MR; ++t) {
    const int r = g + 16 * t;
    col[t] = r < m ? A[(size_t)(c0 + c) * ld + r0 + r] : make_double2(0, 0);
  }
  // the group's rows of column 0 become the first pivot
  if (c == 0) {
#pragma unroll
    for (int t = 0; t < MR; ++t) pv[t] = col[t];
  }
  __syncwarp();
  for (int j = 0; j < kNB; ++j) {
    const int buf = j & 1;
    // ---- partial sums over this thread's rows r > j
    double2 acc = make_double2(0, 0);
#pragma unroll
    for (int t = 0; t < MR; ++t) {
      const int r = g + 16 * t;
      if (r > j && r < m) {
        const double2 aj = pv[t];
        if (c > j)
          acc = cadd(acc, cmulc(aj, col[t]));
        else if (c < j)
          acc = cadd(acc, cmulc(col[t], aj));
        else
          acc.x += aj.x * aj.x + aj.y * aj.y;
      }
    }
    red[(buf * 16 + g) * 16 + c] = acc;
    if (g == j) rowj[buf * 16 + c] = col[0];  // row j = row group j, slot 0
    __syncthreads();
    double2 tot = make_double2(0, 0);
    double xn = 0.0;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      tot = cadd(tot, red[(buf * 16 + q) * 16 + c]);
      xn += red[(buf * 16 + q) * 16 + j].x;
    }
    const double2 alpha = rowj[buf * 16 + j], rj = rowj[buf * 16 + c];
    const Refl R = make_refl(alpha, xn);
    if (c > j) {
      // w_c = conj(tau) v^H a_c; a_c -= v w_c with v = (1; scal a_j)
      const double2 w = cmul(cconj(R.tau), cadd(rj, cmulc(R.scal, tot)));
      const double2 sw = cmul(R.scal, w);
#pragma unroll
      for (int t = 0; t < MR; ++t) {
        const int r = g + 16 * t;
        if (r > j && r < m) col[t] = csub(col[t], cmul(pv[t], sw));
      }
      if (g == j) col[0] = csub(col[0], w);
    } else if (c == j) {
#pragma unroll
      for (int t = 0; t < MR; ++t) {
        const int r = g + 16 * t;
        if (r > j && r < m) col[t] = cmul(col[t], R.scal);
      }
      if (g == j) col[0] = make_double2(R.beta, 0.0);
    } else if (g == 0) {
      dsm[j * 16 + c] = cadd(cconj(rj), cmul(R.scal, tot));  // v_c^H v_j
    }
    if (tid == 0) tsm[j] = R.tau;
    // T column j - 1 (its dots are complete now): T[0:j-1, j-1] = -tau T d
    if (wid == 0 && j >= 1) {
      const int jj = j - 1;
      double2 sacc = make_double2(0, 0);
      if (lane < jj)
        for (int q = lane; q < jj; ++q) sacc = cadd(sacc, cmul(T[lane * 17 + q], dsm[jj * 16 + q]));
      const double2 tj = tsm[jj];
      if (lane < jj) T[lane * 17 + jj] = cmul(make_double2(-tj.x, -tj.y), sacc);
      if (lane == jj) T[jj * 17 + jj] = tj;
      if (lane > jj && lane < kNB) T[lane * 17 + jj] = make_double2(0, 0);
    }
    // the next pivot column reaches the group through the warp's buffer
    __syncwarp();
    if (j + 1 < kNB && c == j + 1) {
#pragma unroll
      for (int t = 0; t < MR; ++t) pv[t] = col[t];
    }
    __syncwarp();
  }
  __syncthreads();
  if (wid == 0) {  // last T column
    const int jj = kNB - 1;
    double2 sacc = make_double2(0, 0);
    if (lane < jj)
      for (int q = lane; q < jj; ++q) sacc = cadd(sacc, cmul(T[lane * 17 + q], dsm[jj * 16 + q]));
    const double2 tj = tsm[jj];
    if (lane < jj) T[lane * 17 + jj] = cmul(make_double2(-tj.x, -tj.y), sacc);
    if (lane == jj) T[jj * 17 + jj] = tj;
  }
  // R and the reflectors back in place (band and back-transform); V explicit
  // in shared memory
#pragma unroll
  for (int t = 0; t < MR; ++t) {
    const int r = g + 16 * t;
    if (r < m) {
      A[(size_t)(c0 + c) * ld + r0 + r] = col[t];
      V[pidx(r, c)] = r < c ? make_double2(0, 0) : (r == c ? make_double2(1, 0) : col[t]);
    }
  }
  __syncthreads();
}

// Y[m x 16] = A22 V: every warp owns 8-row blocks; the upper tiles of the
// Hermitian trailing block are read as conjugate transposes of the lower ones,
// the diagonal tiles (kept full) directly.
__device__ void pass_y(const double2* __restrict__ A, int ld, int r0, int Mt, const double2* V, double2* Y) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int gr = lane >> 2, gk = lane & 3;
  for (int I8 = wid; I8 < 2 * Mt; I8 += kNW) {
    const int I = I8 >> 1;
    const int row = r0 + 8 * I8 + gr;  // this lane's A row
    double cr[2][2], ci[2][2];
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) cr[nb][0] = cr[nb][1] = ci[nb][0] = ci[nb][1] = 0.0;
    double2 a[4], an[4];
    auto load_a = [&](int J, double2 (&f)[4]) {
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
        const int col = r0 + 16 * J + 4 * kb + gk;
        if (I >= J)
          f[kb] = A[(size_t)col * ld + row];
        else
          f[kb] = cconj(A[(size_t)row * ld + col]);
      }
    };
    load_a(0, a);
    for (int J = 0; J < Mt; ++J) {
      if (J + 1 < Mt) load_a(J + 1, an);
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
          const double2 b = V[pidx(16 * J + 4 * kb + gk, 8 * nb + gr)];
          cmma(cr[nb], ci[nb], a[kb], b);
        }
      }
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) a[kb] = an[kb];
    }
#pragma unroll
    for (int nb = 0; nb < 2; ++nb)
#pragma unroll
      for (int i = 0; i < 2; ++i) Y[pidx(8 * I8 + gr, 8 * nb + 2 * gk + i)] = make_double2(cr[nb][i], ci[nb][i]);
  }
}

// A22 -= V X^H + X V^H on the lower 16 x 16 tiles (diagonal tiles in full).
__device__ void pass_u(double2* __restrict__ A, int ld, int r0, int Mt, const double2* V, const double2* X) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int gr = lane >> 2, gk = lane & 3;
  int I = 0, J = wid;
  while (I < Mt && J > I) {  // tile t = wid in lower-triangle order
    J -= I + 1;
    ++I;
  }
  double2 c[2][2][2], cn[2][2][2];
  auto addr = [&](int TI, int TJ, int rb, int nb, int i) {
    return (size_t)(r0 + 16 * TJ + 8 * nb + 2 * gk + i) * ld + (r0 + 16 * TI + 8 * rb + gr);
  };
  auto load_c = [&](int TI, int TJ, double2 (&f)[2][2][2]) {
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
      for (int nb = 0; nb < 2; ++nb)
#pragma unroll
        for (int i = 0; i < 2; ++i) f[rb][nb][i] = A[addr(TI, TJ, rb, nb, i)];
  };
  auto advance = [&](int& TI, int& TJ) {  // 8 tiles further in lower-triangle order
    TJ += kNW;
    while (TI < Mt && TJ > TI) {
      TJ -= TI + 1;
      ++TI;
    }
  };
  if (I < Mt) load_c(I, J, c);
  while (I < Mt) {
    int In = I, Jn = J;
    advance(In, Jn);
    if (In < Mt) load_c(In, Jn, cn);
    double cr[2][2][2], ci[2][2][2];
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
      for (int nb = 0; nb < 2; ++nb)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          cr[rb][nb][i] = c[rb][nb][i].x;
          ci[rb][nb][i] = c[rb][nb][i].y;
        }
#pragma unroll
    for (int kb = 0; kb < 4; ++kb) {
      double2 vi[2], xi[2], vj[2], xj[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        vi[q] = V[pidx(16 * I + 8 * q + gr, 4 * kb + gk)];
        xi[q] = X[pidx(16 * I + 8 * q + gr, 4 * kb + gk)];
        vj[q] = V[pidx(16 * J + 8 * q + gr, 4 * kb + gk)];
        xj[q] = X[pidx(16 * J + 8 * q + gr, 4 * kb + gk)];
      }
#pragma unroll
      for (int rb = 0; rb < 2; ++rb)
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
          cmma_sub_herm(cr[rb][nb], ci[rb][nb], vi[rb], xj[nb]);
          cmma_sub_herm(cr[rb][nb], ci[rb][nb], xi[rb], vj[nb]);
        }
    }
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
      for (int nb = 0; nb < 2; ++nb)
#pragma unroll
        for (int i = 0; i < 2; ++i) A[addr(I, J, rb, nb, i)] = make_double2(cr[rb][nb][i], ci[rb][nb][i]);
    I = In;
    J = Jn;
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
      for (int nb = 0; nb < 2; ++nb)
#pragma unroll
        for (int i = 0; i < 2; ++i) c[rb][nb][i] = cn[rb][nb][i];
  }
}

}  // namespace

template <int MR>
__global__ void __launch_bounds__(kThr, 1) sb_kernel(const EigItem* __restrict__ items, double2* __restrict__ hbuf) {
  const EigItem it = items[blockIdx.x];
  const int ld = it.ld;
  const int tid = threadIdx.x;
  double2* A = hbuf + it.h_off;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int mmax = ld - kNB;
  SbSmem S;
  S.V = reinterpret_cast<double2*>(smraw);
  S.Y = S.V + (size_t)mmax * kNB;
  S.T = S.Y + (size_t)mmax * kNB;
  S.M = S.T + kNB * 17;
  S.P = S.M + kNB * 17;
  S.taus = S.P + kNB * 17;
  S.part = S.Y;  // 512 + 32 + 16 MR <= 16 mmax double2 for ld >= 96
  S.rowj = S.part + 2 * 16 * 16;
  S.pvw = S.rowj + 2 * 16;

  for (int c0 = 0; c0 + kNB < ld; c0 += kNB) {
    const int r0 = c0 + kNB, m = ld - r0, Mt = m / kNB;
    panel_qr<MR>(A, ld, c0, r0, m, S.V, S.T, S.part, S.rowj, S.pvw, S.M, S.taus);
    // T into the free upper tile (rows c0.., columns r0..) for the back-transform
    for (int idx = tid; idx < kNB * kNB; idx += kThr) {
      const int i = idx % kNB, j = idx / kNB;
      A[(size_t)(r0 + j) * ld + c0 + i] = S.T[i * 17 + j];
    }
    // ---- Y = A22 V on the tensor cores
    pass_y(A, ld, r0, Mt, S.V, S.Y);
    __syncthreads();
    // ---- X = Y T - 1/2 V (T^H V^H Y T): Y <- Y T row by row (T upper
    // triangular, columns from the right so that the row can be updated in place)
    for (int r = tid; r < m; r += kThr) {
      double2 y[kNB];
#pragma unroll
      for (int c = 0; c < kNB; ++c) y[c] = S.Y[pidx(r, c)];
#pragma unroll
      for (int c = kNB - 1; c >= 0; --c) {
        double2 s = make_double2(0, 0);
#pragma unroll
        for (int k = 0; k <= c; ++k) s = cadd(s, cmul(y[k], S.T[k * 17 + c]));
        y[c] = s;
      }
#pragma unroll
      for (int c = 0; c < kNB; ++c) S.Y[pidx(r, c)] = y[c];
    }
    __syncthreads();
    {  // M = V^H Y
      const int i = tid / kNB, j = tid % kNB;
      double2 s = make_double2(0, 0);
      for (int r = i; r < m; ++r) s = cadd(s, cmulc(S.V[pidx(r, i)], S.Y[pidx(r, j)]));
      S.M[i * 17 + j] = s;
    }
    __syncthreads();
    {  // P = T^H M
      const int i = tid / kNB, j = tid % kNB;
      double2 s = make_double2(0, 0);
      for (int k = 0; k <= i; ++k) s = cadd(s, cmulc(S.T[k * 17 + i], S.M[k * 17 + j]));
      S.P[i * 17 + j] = s;
    }
    __syncthreads();
    for (int r = tid; r < m; r += kThr) {
      double2 v[kNB];
#pragma unroll
      for (int k = 0; k < kNB; ++k) v[k] = S.V[pidx(r, k)];
#pragma unroll
      for (int c = 0; c < kNB; ++c) {
        double2 s = make_double2(0, 0);
#pragma unroll
        for (int k = 0; k < kNB; ++k) s = cadd(s, cmul(v[k], S.P[k * 17 + c]));
        S.Y[pidx(r, c)] = csub(S.Y[pidx(r, c)], cscale(s, 0.5));
      }
    }
    __syncthreads();
    // ---- A22 -= V X^H + X V^H on the tensor cores
    pass_u(A, ld, r0, Mt, S.V, S.Y);
    __syncthreads();
  }
}

// ------------------------------------------------------------------ stage 2
// Band storage Bd[c * kBandLd + d] = A(c + d, c), d = 0..31: the band and the
// bulge (a task reaches d = len + 15 <= 31 at most). kBandLd is even, so reads
// along a row of the band (stride kBandLd - 1) and down a column (stride 1)
// are both free of bank conflicts.
constexpr int kBandLd = 2 * kNB;
constexpr int kSlots = 10;          // sweeps in flight: at most ceil(26 / 3) = 9 for ld 416
constexpr int kS2Thr = 512;         // 8 tasks x (D warp + E warp)
constexpr int kS2W = kS2Thr / 32;

__host__ __device__ inline size_t sbtrd_smem_bytes(int ld) {
  return sizeof(double2) * ((size_t)ld * kBandLd + kSlots * 17 + kSlots * kNB + kS2W * 2 * kNB) +
         sizeof(double) * kSlots;
}

// Reflector of a 16-vector held as x_i on lanes i (both 16-lane halves hold
// the same values): v_i on lane i (v_0 = 1, zero beyond len), tau, beta.
__device__ __forceinline__ Refl refl16(double2 x, int i, int len, double2& v) {
  const double xn = sum16(i >= 1 && i < len ? x.x * x.x + x.y * x.y : 0.0);
  const double2 a0 = make_double2(__shfl_sync(0xffffffffu, x.x, 0), __shfl_sync(0xffffffffu, x.y, 0));
  const Refl R = make_refl(a0, xn);
  v = i == 0 ? make_double2(1, 0) : (i < len ? cmul(x, R.scal) : make_double2(0, 0));
  return R;
}

__global__ void __launch_bounds__(kS2Thr, 1) sbtrd_kernel(const EigItem* __restrict__ items,
                                                        const double2* __restrict__ hbuf, double2* __restrict__ rbuf) {
  const EigItem it = items[blockIdx.x];
  const int ld = it.ld;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double2* A = hbuf + it.h_off;
  double2* R = rbuf + it.r_off;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* Bd = reinterpret_cast<double2*>(smraw);
  double2* slot = Bd + (size_t)ld * kBandLd;  // [kSlots][17]: v[16], tau of the sweeps in flight
  double2* v2s = slot + kSlots * 17;          // [kSlots][16]: new reflectors (tau in place of v_0)
  double2* wsm = v2s + kSlots * kNB;          // [16 warps][32]: vectors a warp broadcasts to its lanes
  double* bst = reinterpret_cast<double*>(wsm + kS2W * 2 * kNB);  // [kSlots]: beta of a sweep's column
  for (int idx = tid; idx < ld * kBandLd; idx += kS2Thr) {
    const int c = idx / kBandLd, d = idx % kBandLd;
    Bd[idx] = (d <= kNB && c + d < ld) ? A[(size_t)c * ld + c + d] : make_double2(0, 0);
  }
  __syncthreads();
  // A(r, c) for 0 <= r - c <= 31 (int arithmetic, never a negative offset)
  auto at = [&](int r, int c) -> double2& { return Bd[c * kBandLd + (r - c)]; };
  const int i = lane & 15, h = lane >> 4;
  const int pair = wid >> 1;          // task slot of this warp
  const bool ewarp = (wid & 1) != 0;  // E (bulge) warp, else D (diagonal block) warp
  double2* wv = wsm + wid * 2 * kNB;  // [0..15] first vector, [16..31] second
  const int tmax = kLag * (ld - 2);
  for (int t = 0; t <= tmax; ++t) {
    const int smax = min(t / kLag, ld - 2);
    int smin = smax;
    while (smin - 1 >= 0 && t - kLag * (smin - 1) < sweep_steps(ld, smin - 1)) --smin;
    if (t - kLag * smax >= sweep_steps(ld, smax)) smin = smax + 1;  // nothing active
    for (int s = smax - pair; s >= smin; s -= 8) {
      const int j = t - kLag * s;
      const int p = s + 1 + kNB * j, len = min(kNB, ld - p), q = p + len;
      const long long ridx = sweep_first(ld, s);
      // this task's reflector v (16, zero beyond len) and tau into wv[0..15]
      double2 tau;
      const double2* vv;
      if (j == 0) {
        // from column s, rows s+1 .. s+len (both warps; the D warp stages beta
        // and records the reflector)
        double2 v;
        const double2 x = i < len ? at(p + i, s) : make_double2(0, 0);
        const Refl Rf = refl16(x, i, len, v);
        tau = Rf.tau;
        if (h == 0) wv[i] = v;
        if (!ewarp && h == 0) {
          if (i == 0) bst[s % kSlots] = Rf.beta;
          R[ridx * kNB + i] = i == 0 ? tau : v;
        }
        __syncwarp();
        vv = wv;
      } else {
        vv = slot + (s % kSlots) * 17;
        tau = vv[16];
      }
      const double2 vi = vv[i];
      if (!ewarp) {
        // ---- D <- H^H D H on D = A(p : p+len, p : p+len): lane (row i, half h)
        double2 d[8], y = make_double2(0, 0);
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int c = 8 * h + cc;
          // lower triangle directly, upper as the conjugate of the lower:
          // column min(i, c), offset |i - c|
          const int lo = c <= i ? c : i, off = c <= i ? i - c : c - i;
          double2 val = Bd[(p + lo) * kBandLd + off];
          if (c > i) val.y = -val.y;
          d[cc] = (i < len && c < len) ? val : make_double2(0, 0);
        }
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) y = cadd(y, cmul(d[cc], vv[8 * h + cc]));
        y.x += __shfl_xor_sync(0xffffffffu, y.x, 16);
        y.y += __shfl_xor_sync(0xffffffffu, y.y, 16);
        const double vhy = sum16(i < len ? cmulc(vi, y).x : 0.0);
        const double al = -0.5 * (tau.x * tau.x + tau.y * tau.y) * vhy;
        const double2 w = cadd(cmul(tau, y), cscale(vi, al));
        if (h == 0) wv[kNB + i] = w;
        __syncwarp();
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int c = 8 * h + cc;
          if (i < len && c <= i)
            at(p + i, p + c) = csub(d[cc], cadd(cmul(vi, cconj(wv[kNB + c])), cmul(w, cconj(vv[c]))));
        }
      } else if (q < ld) {
        // ---- E = A(q : q+len2, p : p+len) <- E H, then the next reflector
        // from E's first column and E(:, 1:) <- H2^H E(:, 1:)
        const int len2 = min(kNB, ld - q);
        double2 e[8], u = make_double2(0, 0);
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int c = 8 * h + cc;
          e[cc] = (i < len2 && c < len) ? at(q + i, p + c) : make_double2(0, 0);
        }
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) u = cadd(u, cmul(e[cc], vv[8 * h + cc]));
        u.x += __shfl_xor_sync(0xffffffffu, u.x, 16);
        u.y += __shfl_xor_sync(0xffffffffu, u.y, 16);
        const double2 tu = cmul(tau, u);  // E(i, c) -= tau u_i conj(v_c)
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) e[cc] = csub(e[cc], cmul(tu, cconj(vv[8 * h + cc])));
        // E(i, 0) sits on lane (i, half 0); the rows go to shared memory
        if (h == 0) wv[kNB + i] = e[0];
        __syncwarp();
        const double2 x = wv[kNB + i];
        double2 v2;
        const Refl Rf = refl16(x, i, len2, v2);
        if (h == 0) e[0] = i == 0 ? make_double2(Rf.beta, 0) : make_double2(0, 0);
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int c = 8 * h + cc;
          if (i < len2 && c < len) at(q + i, p + c) = e[cc];
        }
        __syncwarp();  // every lane has read wv (x) and stored its row
        if (h == 0) wv[i] = v2;  // (this warp's v was read into registers above)
        __syncwarp();
        // E(:, 1:) <- H2^H E(:, 1:): lane (column c = i, rows of half h)
        const double2 t2 = cconj(Rf.tau);
        const int c = i;
        double2 col[8], zc = make_double2(0, 0);
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
          const int r = 8 * h + rr;
          col[rr] = (c >= 1 && c < len && r < len2) ? at(q + r, p + c) : make_double2(0, 0);
        }
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) zc = cadd(zc, cmulc(wv[8 * h + rr], col[rr]));
        zc.x += __shfl_xor_sync(0xffffffffu, zc.x, 16);
        zc.y += __shfl_xor_sync(0xffffffffu, zc.y, 16);
        const double2 tz = cmul(t2, zc);
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
          const int r = 8 * h + rr;
          if (c >= 1 && c < len && r < len2) at(q + r, p + c) = csub(col[rr], cmul(wv[r], tz));
        }
        if (h == 0) {
          // staged: the D warp of this task may still be reading the sweep's slot
          v2s[(s % kSlots) * kNB + i] = i == 0 ? Rf.tau : v2;
          R[(ridx + j + 1) * kNB + i] = i == 0 ? Rf.tau : v2;
        }
      }
      __syncwarp();  // wv is rewritten by this warp's next task
    }
    __syncthreads();
    // every task of this time step is done: the new reflectors move into
    // their sweeps' slots, and the first task of the newest sweep writes its
    // column (beta, zeros below), which no task of this step read after it
    for (int s = smax - (tid >> 4); s >= smin; s -= kS2Thr / 16) {
      const int j = t - kLag * s;
      const int p = s + 1 + kNB * j, len = min(kNB, ld - p), q = p + len;
      const int k = tid & 15;
      double2* sl = slot + (s % kSlots) * 17;
      if (q < ld) {
        const double2 val = v2s[(s % kSlots) * kNB + k];
        if (k == 0) {
          sl[16] = val;
          sl[0] = make_double2(1, 0);
        } else {
          sl[k] = val;
        }
      }
      if (j == 0 && k < len) at(p + k, s) = k == 0 ? make_double2(bst[s % kSlots], 0) : make_double2(0, 0);
    }
    __syncthreads();
  }
  // tridiagonal T after the reflectors above: d real, e real (beta)
  double* de = reinterpret_cast<double*>(R + ceil_sum(ld - 1) * kNB);
  for (int c = tid; c < ld; c += kS2Thr) {
    de[c] = Bd[(size_t)c * kBandLd].x;
    de[ld + c] = c + 1 < ld ? Bd[(size_t)c * kBandLd + 1].x : 0.0;
  }
}

// --------------------------------------------------------- tridiagonal stage
// 256 threads per matrix (one CTA): multisection bisection probes 256 / nval
// points per eigenvalue at once; the inverse iteration runs one thread per
// eigenvalue cluster (128-thread CTAs measured slower: 1.29 vs 1.16 ms)
constexpr int kTriThr = 256;

__host__ __device__ inline size_t tri_smem_bytes(int n, int nval, int nvec) {
  return sizeof(double) * ((size_t)3 * n + 8 + 3 * nval + kTriThr) + sizeof(int) * ((size_t)kTriThr + nvec + 1 + 4);
}

__global__ void __launch_bounds__(kTriThr) tri_eig_kernel(const EigItem* __restrict__ items,
                                                     const double2* __restrict__ rbuf, double* __restrict__ wbuf,
                                                     double2* __restrict__ zbuf, double* __restrict__ scratch,
                                                     int* __restrict__ info) {
  const EigItem it = items[blockIdx.x];
  const int n = it.n, ld = it.ld, nval = it.nval, nvec = it.want_vec ? it.nev : 0;
  const int tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* d = reinterpret_cast<double*>(smraw);
  double* e = d + n;
  double* e2 = e + n;
  double* red = e2 + n;
  double* lam = red + 8;
  double* lo = lam + nval;
  double* hi = lo + nval;
  double* xs = hi + nval;
  int* cnt = reinterpret_cast<int*>(xs + kTriThr);
  int* clus = cnt + kTriThr;
  int* misc = clus + nvec + 1;
  const double* de = reinterpret_cast<const double*>(rbuf + it.r_off + ceil_sum(ld - 1) * kNB);
  for (int c = tid; c < n; c += kTriThr) {
    d[c] = de[c];
    e[c] = c + 1 < n ? de[ld + c] : 0.0;
  }
  __syncthreads();
  const TriWork tw{d, e, e2, red, lam, lo, hi, xs, cnt, clus, misc};
  const int status = tri_eigvals(tw, n, nval, wbuf + it.w_off, it.bisect_cap);
  if (nvec > 0 && status == 0) tri_eigvecs(tw, n, nvec, zbuf + it.z_off, scratch + it.s_off, blockIdx.x);
  if (tid == 0) info[blockIdx.x] = status;
}

// ----------------------------------------------------------- back-transform
constexpr int kChunk = 32;  // panel rows per staged chunk of the stage-1 back-transform

__host__ __device__ inline size_t back_smem_bytes(int ld, int vb) {
  // Z [ld][vb], one sweep's reflectors [2][ceil(ld/16)][16], panel chunks
  // [2][kChunk][16], W [16][vb], T [16][17]
  return sizeof(double2) *
         ((size_t)ld * vb + 2 * ((ld + kNB - 1) / kNB) * kNB + 2 * kChunk * kNB + kNB * vb + kNB * 17);
}
// eigenvectors per back-transform CTA: up to kVecBlock, and few enough that
// two CTAs share an SM (the stage is latency-bound)
inline int back_vec_block(int ld, int max_nvec) {
  int vb = std::min(kVecBlock, std::max(max_nvec, 1));
  while (vb > 1 && back_smem_bytes(ld, vb) > (size_t)112 * 1024) --vb;
  return vb;
}

__global__ void __launch_bounds__(kThr, 2) eig2_back_kernel(const EigItem* __restrict__ items,
                                                       const double2* __restrict__ hbuf,
                                                       const double2* __restrict__ rbuf, double2* __restrict__ zbuf,
                                                       const int* __restrict__ info, int vb) {
  const EigItem it = items[blockIdx.x];
  const int n = it.n, ld = it.ld, nvec = it.want_vec ? it.nev : 0;
  const int k0 = blockIdx.y * vb;
  if (k0 >= nvec || info[blockIdx.x] != 0) return;
  const int nv = min(vb, nvec - k0);
  const int tid = threadIdx.x;
  const double2* A = hbuf + it.h_off;
  const double2* R = rbuf + it.r_off;
  double2* zg = zbuf + it.z_off;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int maxsteps = (ld + kNB - 1) / kNB;
  double2* Z = reinterpret_cast<double2*>(smraw);  // Z[r * nv + k]
  double2* RB = Z + (size_t)ld * nv;               // [2][maxsteps * 16]
  double2* VC = RB + 2 * maxsteps * kNB;           // [2][64][16]
  double2* W = VC + 2 * kChunk * kNB;              // [16][nv]
  double2* T = W + kNB * nv;                       // [16][17]
  for (int idx = tid; idx < ld * nv; idx += kThr) {
    const int r = idx / nv, k = idx % nv;
    Z[idx] = r < n ? zg[(size_t)(k0 + k) * n + r] : make_double2(0, 0);
  }
  // ---- band reflectors, sweeps in reverse; one sweep's reflectors act on
  // disjoint rows and are applied together (one thread per reflector and
  // vector); the next sweep's reflectors stream in (cp.async) meanwhile
  auto prefetch = [&](int s, double2* dst) {
    const int ns = sweep_steps(ld, s);
    const double2* src = R + sweep_first(ld, s) * kNB;
    for (int idx = tid; idx < ns * kNB; idx += kThr) cp_async16(dst + idx, src + idx);
    cp_async_commit();
  };
  prefetch(ld - 2, RB);
  cp_async_wait<0>();
  __syncthreads();
  for (int s = ld - 2; s >= 0; --s) {
    const double2* cur = RB + ((ld - 2 - s) & 1) * maxsteps * kNB;
    if (s > 0) prefetch(s - 1, RB + ((ld - 1 - s) & 1) * maxsteps * kNB);
    const int ns = sweep_steps(ld, s);
    for (int task = tid; task < ns * nv; task += kThr) {
      const int j = task / nv, k = task % nv;
      const int p = s + 1 + kNB * j, len = min(kNB, ld - p);
      const double2* v = cur + j * kNB;
      const double2 tau = v[0];
      if (tau.x == 0.0 && tau.y == 0.0) continue;
      double2* zc = Z + (size_t)p * nv + k;
      double2 zr[kNB];
#pragma unroll
      for (int q = 0; q < kNB; ++q) zr[q] = q < len ? zc[(size_t)q * nv] : make_double2(0, 0);
      double2 d0 = zr[0], d1 = make_double2(0, 0);
#pragma unroll
      for (int q = 1; q < kNB; q += 2) {
        d1 = cadd(d1, cmulc(v[q], zr[q]));
        if (q + 1 < kNB) d0 = cadd(d0, cmulc(v[q + 1], zr[q + 1]));
      }
      const double2 dot = cmul(tau, cadd(d0, d1));
      zc[0] = csub(zr[0], dot);
#pragma unroll
      for (int q = 1; q < kNB; ++q)
        if (q < len) zc[(size_t)q * nv] = csub(zr[q], cmul(v[q], dot));
    }
    cp_async_wait<0>();
    __syncthreads();
  }
  // ---- panels in reverse: Z[r0:] -= V (T (V^H Z[r0:])); V streams in
  // 64-row chunks (cp.async, double-buffered), explicit unit diagonal
  auto load_chunk = [&](int c0, int r0, int rc, int m, double2* dst) {
    const int rows = min(kChunk, m - rc);
    for (int idx = tid; idx < rows * kNB; idx += kThr) {
      const int r = idx % rows, c = idx / rows;
      cp_async16(dst + r * kNB + c, A + (size_t)(c0 + c) * ld + r0 + rc + r);
    }
    cp_async_commit();
  };
  auto fix_chunk = [&](int rc, int rows, double2* dst) {  // rows < 16 of the panel: unit diagonal, zeros above
    if (rc > 0) return;
    for (int idx = tid; idx < kNB * kNB; idx += kThr) {
      const int r = idx / kNB, c = idx % kNB;
      if (r < rows && r <= c) dst[r * kNB + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    }
  };
  for (int c0 = ld - 2 * kNB; c0 >= 0; c0 -= kNB) {
    const int r0 = c0 + kNB, m = ld - r0, nch = (m + kChunk - 1) / kChunk;
    for (int idx = tid; idx < kNB * kNB; idx += kThr) {
      const int i = idx % kNB, j = idx / kNB;
      T[i * 17 + j] = A[(size_t)(r0 + j) * ld + c0 + i];
    }
    // W = V^H Z[r0:]: thread (i, k) over the chunks
    double2 wacc[2][2] = {{make_double2(0, 0), make_double2(0, 0)}, {make_double2(0, 0), make_double2(0, 0)}};
    load_chunk(c0, r0, 0, m, VC);
    for (int ch = 0; ch < nch; ++ch) {
      double2* cur = VC + (ch & 1) * kChunk * kNB;
      if (ch + 1 < nch) load_chunk(c0, r0, (ch + 1) * kChunk, m, VC + ((ch + 1) & 1) * kChunk * kNB);
      if (ch + 1 < nch) cp_async_wait<1>(); else cp_async_wait<0>();
      __syncthreads();
      const int rows = min(kChunk, m - ch * kChunk);
      fix_chunk(ch * kChunk, rows, cur);
      __syncthreads();
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        const int idx = tid + o * kThr;
        if (idx < kNB * nv) {
          const int i = idx / nv, k = idx % nv;
          const double2* zc = Z + (size_t)(r0 + ch * kChunk) * nv + k;
          for (int r = 0; r < rows; r += 2) {
            wacc[o][0] = cadd(wacc[o][0], cmulc(cur[r * kNB + i], zc[(size_t)r * nv]));
            if (r + 1 < rows) wacc[o][1] = cadd(wacc[o][1], cmulc(cur[(r + 1) * kNB + i], zc[(size_t)(r + 1) * nv]));
          }
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      const int idx = tid + o * kThr;
      if (idx < kNB * nv) W[idx] = cadd(wacc[o][0], wacc[o][1]);
    }
    __syncthreads();
    // W <- T W (T upper triangular): thread per column k
    for (int k = tid; k < nv; k += kThr) {
      double2 w[kNB];
#pragma unroll
      for (int i = 0; i < kNB; ++i) w[i] = W[i * nv + k];
#pragma unroll
      for (int i = 0; i < kNB; ++i) {
        double2 s = make_double2(0, 0);
#pragma unroll
        for (int q = i; q < kNB; ++q) s = cadd(s, cmul(T[i * 17 + q], w[q]));
        W[i * nv + k] = s;
      }
    }
    // Z[r0:] -= V W
    load_chunk(c0, r0, 0, m, VC);
    for (int ch = 0; ch < nch; ++ch) {
      double2* cur = VC + (ch & 1) * kChunk * kNB;
      if (ch + 1 < nch) load_chunk(c0, r0, (ch + 1) * kChunk, m, VC + ((ch + 1) & 1) * kChunk * kNB);
      if (ch + 1 < nch) cp_async_wait<1>(); else cp_async_wait<0>();
      __syncthreads();
      const int rows = min(kChunk, m - ch * kChunk);
      fix_chunk(ch * kChunk, rows, cur);
      __syncthreads();
      for (int idx = tid; idx < rows * nv; idx += kThr) {
        const int r = idx / nv, k = idx % nv;
        double2 s0 = make_double2(0, 0), s1 = make_double2(0, 0);
#pragma unroll
        for (int i = 0; i < kNB; i += 2) {
          s0 = cadd(s0, cmul(cur[r * kNB + i], W[i * nv + k]));
          s1 = cadd(s1, cmul(cur[r * kNB + i + 1], W[(i + 1) * nv + k]));
        }
        double2* z = Z + (size_t)(r0 + ch * kChunk + r) * nv + k;
        *z = csub(*z, cadd(s0, s1));
      }
      __syncthreads();
    }
  }
  for (int idx = tid; idx < n * nv; idx += kThr) {
    const int k = idx / n, r = idx % n;
    zg[(size_t)(k0 + k) * n + r] = Z[(size_t)r * nv + k];
  }
}

// ------------------------------------------------------------------- host
int heev2_ld(int n) { return (n + kNB - 1) / kNB * kNB; }

bool heev2_supported(int max_n) { return heev2_ld(max_n) >= 96 && heev2_ld(max_n) <= kMaxLd; }

size_t heev2_rbuf_double2(int ld) { return (size_t)ceil_sum(ld - 1) * kNB + (size_t)ld; }

cudaError_t launch_heev2(const EigItem* items, int nitems, int max_n, int max_nval, int max_nvec, double2* hbuf,
                         double* wbuf, double2* zbuf, double* scratch, double2* rbuf, int* info, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  if (!heev2_supported(max_n)) return cudaErrorInvalidValue;
  const int ld = heev2_ld(max_n);
  cudaError_t e;
  const int mr = sb_rows(ld);
  const size_t s1 = sb_smem_bytes(ld);
  auto sb = mr == 9 ? sb_kernel<9> : (mr == 17 ? sb_kernel<17> : sb_kernel<25>);
  e = cudaFuncSetAttribute(sb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1);
  if (e != cudaSuccess) return e;
  sb<<<nitems, kThr, s1, st>>>(items, hbuf);
  const size_t s2 = sbtrd_smem_bytes(ld);
  e = cudaFuncSetAttribute(sbtrd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2);
  if (e != cudaSuccess) return e;
  sbtrd_kernel<<<nitems, kS2Thr, s2, st>>>(items, hbuf, rbuf);
  const size_t s3 = tri_smem_bytes(max_n, max_nval, max_nvec);
  e = cudaFuncSetAttribute(tri_eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s3);
  if (e != cudaSuccess) return e;
  tri_eig_kernel<<<nitems, kTriThr, s3, st>>>(items, rbuf, wbuf, zbuf, scratch, info);
  if (max_nvec > 0) {
    const int vb = back_vec_block(ld, max_nvec);
    const size_t s4 = back_smem_bytes(ld, vb);
    e = cudaFuncSetAttribute(eig2_back_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s4);
    if (e != cudaSuccess) return e;
    eig2_back_kernel<<<dim3(nitems, (max_nvec + vb - 1) / vb), kThr, s4, st>>>(items, hbuf, rbuf, zbuf, info, vb);
  }
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmx
