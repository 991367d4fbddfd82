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
//     Up to ld = 416 the panel V and Y live in shared memory; beyond that
//     (ld <= 800) Y lives in the item's slot of the reflector buffer (L2),
//     and beyond ld = 800 (ld <= 1216) V as well.
//  2. sbtrd_kernel (one CTA per matrix): the band (16 sub-diagonals plus 16
//     for the bulge) lives in shared memory up to ld = 416, beyond that in
//     the item's slot of the reflector buffer (L1/L2); sweeps chase their bulges down
//     the band, eight at a time (a pair of warps per sweep), each step of a
//     sweep waiting only for the previous sweep to leave its rows (progress
//     words in shared memory, no block-wide barrier). Reflectors go to
//     global memory.
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
#include <climits>
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
constexpr int kMaxLd = 1216;   // largest padded dimension
constexpr int kVSmemLd = 800;  // largest one whose stage-1 V fits in shared memory
constexpr int kSmemLd = 416;   // largest one whose stage-1 Y and stage-2 band fit in shared memory
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
// Slot of an item in the reflector buffer (double2 offsets): the band
// reflectors [ceil_sum(ld - 1)][16], the tridiagonal (2 ld doubles), and, in
// launches with ld > kSmemLd, a work area of 32 ld double2: stage 1's Y
// (16 (ld - 16)) and, for ld > kVSmemLd, V after it (16 (ld - 16)); then
// stage 2's band (32 ld).
__host__ __device__ __forceinline__ long long band_off(int ld) { return ceil_sum(ld - 1) * kNB + ld; }

// ------------------------------------------------------------------ stage 1
struct SbSmem {
  double2* V;     // [mmax * 16] panel / reflectors V (explicit unit lower trapezoid)
  double2* Y;     // [mmax * 16] Y = A V, then X
  double2* T;     // [16 * 17]
  double2* M;     // [16 * 17] V^H Y (the panel QR's T dots before that)
  double2* P;     // [16 * 17] T^H M
  double2* taus;  // [16]
  // panel QR work arrays, inside Y (free until Y = A V is formed)
  double2* part;  // [2][8][16] partial sums of the panel QR
  double2* rowj;  // [2][16] the current row of the panel QR
  double2* pvw;   // [8][2][MR] per-warp pivot buffers of the panel QR
};

// register rows per thread of the panel QR for a padded dimension ld
inline int sb_rows(int ld) {
  return ld <= 160 ? 9 : (ld <= 288 ? 17 : (ld <= 416 ? 25 : (ld <= 592 ? 36 : (ld <= 800 ? 49 : 75))));
}

// double2 of the panel QR's work arrays (red, rowj, pvw)
__host__ __device__ inline int sb_qr_work(int mr) { return 2 * 8 * 16 + 2 * 16 + 16 * mr; }
// V [mmax][16] (unless in global memory); then Y [mmax][16] in shared
// memory, or (Y in global memory) the panel QR's work arrays after the
// T/M/P/tau block (ld = 800: 231 KB)
__host__ __device__ inline size_t sb_smem_bytes(int ld, int mr, bool yg, bool vg) {
  const int mmax = ld - kNB;
  return sizeof(double2) * ((vg ? 0 : (size_t)mmax * kNB) + (yg ? (size_t)sb_qr_work(mr) : (size_t)mmax * kNB) +
                            3 * kNB * 17 + kNB);
}

// Householder QR of the m x 16 panel (rows r0.. of columns c0..c0+15 of A)
// and its compact WY factor T; leaves R and the reflectors in A (LAPACK
// layout: R on and above the diagonal, v below it) and the explicit V (unit
// diagonal, zeros above) in shared memory. Thread (column c = tid % 16,
// row group g = tid / 16) holds rows g, g + 16, ... of column c in registers.
// Per column j one CTA-wide reduction of one value per thread, the same
// product for every column, sum_{r > j} conj(a_j[r]) a_c[r]: for c > j it
// gives v^H a_c once the reflector's scale is known, for c = j the norm
// |x|^2, for c < j (conjugated) the dot v_c^H v_j of the T column (zlarft).
// The two row groups of a warp are summed with one shuffle, the eight warps'
// sums in shared memory. The update of the columns has one form for every
// column, a_c[r] -= a_j[r] s_c (s_c = scal w_c for c > j, 1 - scal for c = j,
// 0 for c < j), so that the lanes of a warp do not diverge. T column j - 1 is
// formed in iteration j by all warps, two rows each. The pivot column reaches
// the threads of a row group through the warp's own shared-memory buffer (the
// group's 16 threads share a warp). red/rowj: [2][8][16] / [2][16]; pvw
// [8][2][MR]; dsm [16][16]; tsm [16]; T [16][17].
template <int MR>
__device__ void panel_qr(double2* __restrict__ A, int ld, int c0, int r0, int m, double2* V, double2* T,
                         double2* red, double2* rowj, double2* pvw, double2* dsm, double2* tsm) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int c = tid & 15, g = tid >> 4;
  const int Mt = m / kNB;  // m is a multiple of 16: row slots t < Mt are inside the panel
  double2* pv = pvw + (size_t)wid * 2 * MR + (g & 1) * MR;  // this group's pivot buffer
  double2 col[MR];
#pragma unroll
  for (int t = 0; t < MR; ++t) col[t] = t < Mt ? A[(size_t)(c0 + c) * ld + r0 + g + 16 * t] : make_double2(0, 0);
  // the group's rows of column 0 become the first pivot
  if (c == 0) {
#pragma unroll
    for (int t = 0; t < MR; ++t) pv[t] = col[t];
  }
  __syncwarp();
  for (int j = 0; j < kNB; ++j) {
    const int buf = j & 1;
    // ---- partial sums over this thread's rows r > j (two chains)
    double2 acc0 = make_double2(0, 0), acc1 = make_double2(0, 0);
    if (g > j) {
      const double2 aj = pv[0];
      acc0.x = aj.x * col[0].x + aj.y * col[0].y;
      acc0.y = aj.x * col[0].y - aj.y * col[0].x;
    }
#pragma unroll
    for (int t = 1; t < MR; ++t) {
      if (t < Mt) {
        const double2 aj = pv[t];
        double2& a = (t & 1) ? acc1 : acc0;
        a.x = fma(aj.x, col[t].x, fma(aj.y, col[t].y, a.x));
        a.y = fma(aj.x, col[t].y, fma(-aj.y, col[t].x, a.y));
      }
    }
    double2 acc = cadd(acc0, acc1);
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 16);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 16);
    if (lane < 16) red[(buf * 8 + wid) * 16 + c] = acc;
    if (g == j) rowj[buf * 16 + c] = col[0];  // row j = row group j, slot 0
    __syncthreads();
    double2 tq[8];
    double xq[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      tq[q] = red[(buf * 8 + q) * 16 + c];
      xq[q] = red[(buf * 8 + q) * 16 + j].x;
    }
    const double2 tot = cadd(cadd(cadd(tq[0], tq[1]), cadd(tq[2], tq[3])), cadd(cadd(tq[4], tq[5]), cadd(tq[6], tq[7])));
    const double xn = ((xq[0] + xq[1]) + (xq[2] + xq[3])) + ((xq[4] + xq[5]) + (xq[6] + xq[7]));
    const double2 alpha = rowj[buf * 16 + j], rj = rowj[buf * 16 + c];
    // T column j - 1 (its dots are complete now): T[0:j-1, j-1] = -tau T d,
    // rows 2 wid and 2 wid + 1
    if (j >= 1) {
      const int jj = j - 1, l = 2 * wid + (lane >> 4);
      double2 p = c >= l && c < jj ? cmul(T[l * 17 + c], dsm[jj * 16 + c]) : make_double2(0, 0);
      p.x = sum16(p.x);
      p.y = sum16(p.y);
      const double2 tj = tsm[jj];
      if (c == 0) T[l * 17 + jj] = l < jj ? cmul(make_double2(-tj.x, -tj.y), p) : (l == jj ? tj : make_double2(0, 0));
    }
    const Refl R = make_refl(alpha, xn);
    // w_c = conj(tau) v^H a_c (v = (1; scal a_j)); a_c -= v w_c
    const double2 w = cmul(cconj(R.tau), cadd(rj, cmulc(R.scal, tot)));
    const double2 sw = c > j ? cmul(R.scal, w) : (c == j ? make_double2(1.0 - R.scal.x, -R.scal.y) : make_double2(0, 0));
    if (g > j) col[0] = csub(col[0], cmul(pv[0], sw));
#pragma unroll
    for (int t = 1; t < MR; ++t)
      if (t < Mt) col[t] = csub(col[t], cmul(pv[t], sw));
    if (g == j) col[0] = c > j ? csub(col[0], w) : (c == j ? make_double2(R.beta, 0.0) : col[0]);
    if (g == 0 && c < j) dsm[j * 16 + c] = cadd(cconj(rj), cmul(R.scal, cconj(tot)));  // v_c^H v_j
    if (tid == 0) tsm[j] = R.tau;
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
    if (t < Mt) {
      A[(size_t)(c0 + c) * ld + r0 + r] = col[t];
      V[pidx(r, c)] = r < c ? make_double2(0, 0) : (r == c ? make_double2(1, 0) : col[t]);
    }
  }
  __syncthreads();
}

// Y[m x 16] = A22 V: every warp owns 8-row blocks; the upper tiles of the
// Hermitian trailing block are read as conjugate transposes of the lower ones,
// the diagonal tiles (kept full) directly.
// PF: V in global memory, its fragments of column block J + 1 loaded while
// block J is multiplied
template <bool PF>
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
    double2 bf[4][2], bfn[4][2];
    auto load_b = [&](int J, double2 (&f)[4][2]) {
#pragma unroll
      for (int kb = 0; kb < 4; ++kb)
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) f[kb][nb] = V[pidx(16 * J + 4 * kb + gk, 8 * nb + gr)];
    };
    load_a(0, a);
    if (PF) load_b(0, bf);
    for (int J = 0; J < Mt; ++J) {
      if (J + 1 < Mt) {
        load_a(J + 1, an);
        if (PF) load_b(J + 1, bfn);
      }
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
          const double2 b = PF ? bf[kb][nb] : V[pidx(16 * J + 4 * kb + gk, 8 * nb + gr)];
          cmma(cr[nb], ci[nb], a[kb], b);
        }
      }
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
        a[kb] = an[kb];
        if (PF) {
#pragma unroll
          for (int nb = 0; nb < 2; ++nb) bf[kb][nb] = bfn[kb][nb];
        }
      }
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

// Load of Y in global memory kept in program order: with plain loads the
// compiler hoists the rows' loads of the Y T and P passes far enough ahead to
// spill ~4 KB of the stage's registers
__device__ __forceinline__ double2 ld_ordered(const double2* p) {
  double2 v;
  asm volatile("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p) : "memory");
  return v;
}
template <bool KYG>
__device__ __forceinline__ double2 ldy(const double2* p) {
  return KYG ? ld_ordered(p) : *p;
}

// KYG: Y in the item's work area of the reflector buffer (ld > kSmemLd);
// KVG: V there too (ld > kVSmemLd)
template <int MR, bool KYG, bool KVG = false>
__global__ void __launch_bounds__(kThr, 1) sb_kernel(const EigItem* __restrict__ items, double2* __restrict__ hbuf,
                                                    double2* __restrict__ rbuf) {
  const EigItem it = items[blockIdx.x];
  const int ld = it.ld;
  const int tid = threadIdx.x;
  double2* A = hbuf + it.h_off;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int mmax = ld - kNB;
  SbSmem S;
  double2* work = rbuf + it.r_off + band_off(ld);
  S.V = KVG ? work + (size_t)mmax * kNB : reinterpret_cast<double2*>(smraw);
  S.Y = KYG ? work : S.V + (size_t)mmax * kNB;
  S.T = KVG ? reinterpret_cast<double2*>(smraw) : (KYG ? S.V : S.Y) + (size_t)mmax * kNB;
  S.M = S.T + kNB * 17;
  S.P = S.M + kNB * 17;
  S.taus = S.P + kNB * 17;
  // the panel QR's work arrays: inside Y (free until Y = A V is formed;
  // 256 + 32 + 16 MR <= 16 mmax double2 for ld >= 96), or after taus
  S.part = KYG ? S.taus + kNB : S.Y;
  S.rowj = S.part + 2 * 8 * 16;
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
    pass_y<KVG>(A, ld, r0, Mt, S.V, S.Y);
    __syncthreads();
    // ---- X = Y T - 1/2 V (T^H V^H Y T) on the tensor cores. X1 = Y T in
    // place: a warp owns 8-row blocks of Y (A fragments: its rows; B: T);
    // the lanes' reads of a block end before its writes (__syncwarp)
    {
      const int lane = tid & 31, wid = tid >> 5, gr = lane >> 2, gk = lane & 3;
      for (int I8 = wid; I8 < 2 * Mt; I8 += kNW) {
        double cr[2][2] = {{0, 0}, {0, 0}}, ci[2][2] = {{0, 0}, {0, 0}};
#pragma unroll
        for (int kb = 0; kb < 4; ++kb) {
          const double2 a = ldy<KYG>(S.Y + pidx(8 * I8 + gr, 4 * kb + gk));
#pragma unroll
          for (int nb = 0; nb < 2; ++nb) cmma(cr[nb], ci[nb], a, S.T[(4 * kb + gk) * 17 + 8 * nb + gr]);
        }
        __syncwarp();
#pragma unroll
        for (int nb = 0; nb < 2; ++nb)
#pragma unroll
          for (int i = 0; i < 2; ++i) S.Y[pidx(8 * I8 + gr, 8 * nb + 2 * gk + i)] = make_double2(cr[nb][i], ci[nb][i]);
      }
      __syncthreads();
      // M = V^H X1: warp w computes the 8 x 8 block (w & 3) of M over one half
      // of the rows (w >> 2); the second half's partials pass through P (free
      // until P = T^H M) and are added by the first half's warps in a fixed
      // order
      {
        const int ib = (wid & 3) >> 1, jb = wid & 1, half = wid >> 2;
        double cr[2] = {0, 0}, ci[2] = {0, 0};
        for (int kb = half * 2 * Mt; kb < (half + 1) * 2 * Mt; ++kb) {
          const int k = 4 * kb + gk;
          const double2 a = cconj(ldy<KVG>(S.V + pidx(k, 8 * ib + gr)));
          const double2 b = ldy<KYG>(S.Y + pidx(k, 8 * jb + gr));
          cmma(cr, ci, a, b);
        }
        const int mi = 8 * ib + gr;
        if (half == 1) {
#pragma unroll
          for (int i = 0; i < 2; ++i) S.P[mi * 17 + 8 * jb + 2 * gk + i] = make_double2(cr[i], ci[i]);
        }
        __syncthreads();
        if (half == 0) {
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const double2 o = S.P[mi * 17 + 8 * jb + 2 * gk + i];
            S.M[mi * 17 + 8 * jb + 2 * gk + i] = make_double2(cr[i] + o.x, ci[i] + o.y);
          }
        }
      }
      __syncthreads();
      {  // P = T^H M
        const int i = tid / kNB, j = tid % kNB;
        double2 sacc = make_double2(0, 0);
        for (int k = 0; k <= i; ++k) sacc = cadd(sacc, cmulc(S.T[k * 17 + i], S.M[k * 17 + j]));
        S.P[i * 17 + j] = sacc;
      }
      __syncthreads();
      // X = X1 - 1/2 V P: each lane updates the entries of its own D fragment
      for (int I8 = wid; I8 < 2 * Mt; I8 += kNW) {
        double cr[2][2] = {{0, 0}, {0, 0}}, ci[2][2] = {{0, 0}, {0, 0}};
#pragma unroll
        for (int kb = 0; kb < 4; ++kb) {
          const double2 a = ldy<KVG>(S.V + pidx(8 * I8 + gr, 4 * kb + gk));
#pragma unroll
          for (int nb = 0; nb < 2; ++nb) cmma(cr[nb], ci[nb], a, S.P[(4 * kb + gk) * 17 + 8 * nb + gr]);
        }
#pragma unroll
        for (int nb = 0; nb < 2; ++nb)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            double2* y = S.Y + pidx(8 * I8 + gr, 8 * nb + 2 * gk + i);
            const double2 x1 = ldy<KYG>(y);
            *y = make_double2(x1.x - 0.5 * cr[nb][i], x1.y - 0.5 * ci[nb][i]);
          }
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
//
// Task (s, j) (sweep s, step j, first row p = s + 1 + 16 j) reads and writes
// exactly the elements (r, c) with p <= c < p + 16 and c <= r < p + 32 (its
// diagonal block D and the block E below it), plus column s when j = 0. Two
// tasks of different sweeps commute unless those sets meet, and task (s, j)
// meets sweep s - 1 only in its steps j' <= j + 1. So sweep s may run step j
// as soon as sweep s - 1 has finished min(j + 2, its step count) steps: each
// pair of warps runs its sweeps s = pair, pair + 8, ... and publishes its
// progress in a shared-memory word (release), which the next sweep's pair
// waits for (acquire, bounded by a time limit). No block-wide barrier runs
// between steps.
constexpr int kBandLd = 2 * kNB;
constexpr int kPairs = 8;                // sweeps in flight: one per pair of warps
constexpr int kS2Thr = 64 * kPairs;      // a D warp and an E warp per pair
constexpr int kS2W = kS2Thr / 32;
constexpr int kProgStride = 64;          // progress word: sweep * 64 + steps done (<= 26)
constexpr long long kWaitNs = 2000000000LL;  // default limit of one wait

__host__ __device__ inline size_t sbtrd_smem_bytes(int ld, bool bg) {
  return sizeof(double2) * ((bg ? 0 : (size_t)ld * kBandLd) + kPairs * 2 * 17 + kS2W * 2 * kNB) +
         sizeof(int) * (kPairs + 4);
}

__device__ __forceinline__ int ld_acquire_shared(const int* p) {
  int v;
  asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];"
               : "=r"(v)
               : "r"((unsigned)__cvta_generic_to_shared(p))
               : "memory");
  return v;
}
__device__ __forceinline__ void st_release_shared(int* p, int v) {
  asm volatile("st.release.cta.shared::cta.b32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "r"(v)
               : "memory");
}
__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits until *flag >= need, polling every ~kPollNs so that a waiting warp
// leaves the issue slots to the warps that work. Gives up, and sets *err,
// after limit_ns, after 2^28 polls, or at once when another warp has given
// up already.
constexpr unsigned kPollNs = 40;
__device__ __forceinline__ void wait_progress(const int* flag, int need, int* err, long long limit_ns) {
  if (ld_acquire_shared(flag) >= need) return;
  const long long t0 = global_ns();
  for (int k = 1; k < (1 << 28); ++k) {
    __nanosleep(kPollNs);
    if (ld_acquire_shared(flag) >= need) return;
    if ((k & 63) == 0) {
      if (*reinterpret_cast<volatile int*>(err)) return;
      if (global_ns() - t0 > limit_ns) break;
    }
  }
  atomicExch(err, 1);
}

// KBG: the band in the item's work area of the reflector buffer (ld >
// kSmemLd; a CTA-private region, so the same CTA-scope ordering as in shared
// memory applies)
template <bool KBG>
__global__ void __launch_bounds__(kS2Thr, 1) sbtrd_kernel(const EigItem* __restrict__ items,
                                                        const double2* __restrict__ hbuf, double2* __restrict__ rbuf) {
  const EigItem it = items[blockIdx.x];
  const int ld = it.ld;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double2* A = hbuf + it.h_off;
  double2* R = rbuf + it.r_off;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* Bd = KBG ? R + band_off(ld) : reinterpret_cast<double2*>(smraw);
  // [pair][2][17]: v (v_0 = 1), tau of the pair's next steps
  double2* slots = KBG ? reinterpret_cast<double2*>(smraw) : Bd + (size_t)ld * kBandLd;
  double2* wsm = slots + kPairs * 2 * 17;       // [warp][32]: [0, 16) v, [16, 32) vectors broadcast in a warp
  int* prog = reinterpret_cast<int*>(wsm + kS2W * 2 * kNB);  // [pair]: progress words
  int* err = prog + kPairs;                                  // a wait gave up
  for (int idx = tid; idx < ld * kBandLd; idx += kS2Thr) {
    const int c = idx / kBandLd, d = idx % kBandLd;
    Bd[idx] = (d <= kNB && c + d < ld) ? A[(size_t)c * ld + c + d] : make_double2(0, 0);
  }
  if (tid < kPairs) prog[tid] = -1;
  if (tid == 0) *err = 0;
  __syncthreads();
  // A(r, c) for 0 <= r - c <= 31 (int arithmetic, never a negative offset)
  auto at = [&](int r, int c) -> double2& { return Bd[c * kBandLd + (r - c)]; };
  const int i = lane & 15, h = lane >> 4;
  const int pair = wid >> 1;
  const bool ewarp = (wid & 1) != 0;  // E (bulge) warp, else D (diagonal block) warp
  double2* wv = wsm + wid * 2 * kNB;
  double2* sl = slots + pair * 2 * 17;
  const long long limit = it.wait_ns > 0 ? it.wait_ns : kWaitNs;
  for (int s = pair; s <= ld - 2; s += kPairs) {
    const int ns = sweep_steps(ld, s), nprev = s > 0 ? sweep_steps(ld, s - 1) : 0;
    const long long ridx = sweep_first(ld, s);
    for (int j = 0; j < ns; ++j) {
      const int p = s + 1 + kNB * j, len = min(kNB, ld - p), q = p + len;
      if (s > 0) {  // sweep s - 1 has left the rows of this task
        const int need = (it.wait_fault && s == 1) ? INT_MAX : (s - 1) * kProgStride + min(j + 2, nprev);
        wait_progress(&prog[(s - 1) % kPairs], need, err, limit);
        __syncwarp();
      }
      // this step's reflector: tau, v (all 16 entries at vsrc, v_0 = 1, zero
      // beyond len), v_i and v at this lane's columns 8h .. 8h + 7
      double2 tau, vi, vc[8];
      double beta = 0.0;
      const double2* vsrc;
      if (j == 0) {
        // from column s, rows p .. p + len - 1 (both warps)
        const double2* cs = Bd + (size_t)s * kBandLd + 1;  // A(p + k, s) = cs[k]
        // |x_1..|^2 over the 16 lanes of a half (lane i holds cs[i])
        const double2 xi = i < len ? cs[i] : make_double2(0, 0);
        double xx = i >= 1 ? xi.x * xi.x + xi.y * xi.y : 0.0;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) xx += __shfl_xor_sync(0xffffffffu, xx, o);
        const Refl Rf = make_refl(cs[0], xx);
        tau = Rf.tau;
        beta = Rf.beta;
        vi = i == 0 ? make_double2(1, 0) : (i < len ? cmul(xi, Rf.scal) : make_double2(0, 0));
        if (h == 0) wv[i] = vi;
        if (!ewarp && h == 0) R[ridx * kNB + i] = i == 0 ? tau : vi;
        __syncwarp();
        vsrc = wv;
      } else {
        vsrc = sl + (j & 1) * 17;
        tau = vsrc[16];
        vi = vsrc[i];
      }
#pragma unroll
      for (int cc = 0; cc < 8; ++cc) vc[cc] = vsrc[8 * h + cc];
      if (!ewarp) {
        // ---- D <- H^H D H on D = A(p : p+len, p : p+len): lane (row i, half h)
        double2 d[8];
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
        double2 y0 = make_double2(0, 0), y1 = make_double2(0, 0);
#pragma unroll
        for (int cc = 0; cc < 8; cc += 2) {
          y0 = cadd(y0, cmul(d[cc], vc[cc]));
          y1 = cadd(y1, cmul(d[cc + 1], vc[cc + 1]));
        }
        double2 y = cadd(y0, y1);
        y.x += __shfl_xor_sync(0xffffffffu, y.x, 16);
        y.y += __shfl_xor_sync(0xffffffffu, y.y, 16);
        if (h == 0) wv[kNB + i] = y;
        // v^H y = v^H D v (real; lane i holds row i's term, summed over the
        // half's 16 lanes), w = tau y - 1/2 |tau|^2 (v^H y) v
        double vy = vi.x * y.x + vi.y * y.y;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) vy += __shfl_xor_sync(0xffffffffu, vy, o);
        __syncwarp();
        const double al = -0.5 * (tau.x * tau.x + tau.y * tau.y) * vy;
        const double2 w = cadd(cmul(tau, y), cscale(vi, al));
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int c = 8 * h + cc;
          const double2 wc = cadd(cmul(tau, wv[kNB + c]), cscale(vc[cc], al));
          if (i < len && c <= i) at(p + i, p + c) = csub(d[cc], cadd(cmul(vi, cconj(wc)), cmul(w, cconj(vc[cc]))));
        }
      } else if (q < ld) {
        // ---- E = A(q : q+len2, p : p+len) <- E H, then the next reflector
        // from E's first column and E(:, 1:) <- H2^H E(:, 1:)
        const int len2 = min(kNB, ld - q);
        double2 e[8];
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int c = 8 * h + cc;
          e[cc] = (i < len2 && c < len) ? at(q + i, p + c) : make_double2(0, 0);
        }
        double2 u0 = make_double2(0, 0), u1 = make_double2(0, 0);
#pragma unroll
        for (int cc = 0; cc < 8; cc += 2) {
          u0 = cadd(u0, cmul(e[cc], vc[cc]));
          u1 = cadd(u1, cmul(e[cc + 1], vc[cc + 1]));
        }
        double2 u = cadd(u0, u1);
        u.x += __shfl_xor_sync(0xffffffffu, u.x, 16);
        u.y += __shfl_xor_sync(0xffffffffu, u.y, 16);
        const double2 tu = cmul(tau, u);  // E(i, c) -= tau u_i conj(v_c)
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) e[cc] = csub(e[cc], cmul(tu, cconj(vc[cc])));
        // E's first column x (lane (i, half 0) holds x_i) to every lane
        if (h == 0) wv[kNB + i] = e[0];
        // |x_1..|^2: lane (i, half 0) holds x_i = e[0] (zero for i >= len2)
        double xx = (h == 0 && i >= 1) ? e[0].x * e[0].x + e[0].y * e[0].y : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) xx += __shfl_xor_sync(0xffffffffu, xx, o);
        __syncwarp();
        const Refl Rf = make_refl(wv[kNB], xx);
        if (h == 0) e[0] = i == 0 ? make_double2(Rf.beta, 0) : make_double2(0, 0);
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          const int c = 8 * h + cc;
          if (i < len2 && c < len) at(q + i, p + c) = e[cc];
        }
        __syncwarp();
        // E(:, 1:) <- H2^H E(:, 1:): lane (column c = i, rows of half h);
        // v2_r = x_r scal (v2_0 = 1)
        const double2 t2 = cconj(Rf.tau);
        const int c = i;
        double2 col[8], v2r[8];
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
          const int r = 8 * h + rr;
          col[rr] = (c >= 1 && c < len && r < len2) ? at(q + r, p + c) : make_double2(0, 0);
          v2r[rr] = r == 0 ? make_double2(1, 0) : (r < len2 ? cmul(wv[kNB + r], Rf.scal) : make_double2(0, 0));
        }
        double2 z0 = make_double2(0, 0), z1 = make_double2(0, 0);
#pragma unroll
        for (int rr = 0; rr < 8; rr += 2) {
          z0 = cadd(z0, cmulc(v2r[rr], col[rr]));
          z1 = cadd(z1, cmulc(v2r[rr + 1], col[rr + 1]));
        }
        double2 zc = cadd(z0, z1);
        zc.x += __shfl_xor_sync(0xffffffffu, zc.x, 16);
        zc.y += __shfl_xor_sync(0xffffffffu, zc.y, 16);
        const double2 tz = cmul(t2, zc);
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
          const int r = 8 * h + rr;
          if (c >= 1 && c < len && r < len2) at(q + r, p + c) = csub(col[rr], cmul(v2r[rr], tz));
        }
        if (h == 0) {
          // the pair's next step reads the other slot buffer
          const double2 v2 = i == 0 ? make_double2(1, 0) : (i < len2 ? cmul(wv[kNB + i], Rf.scal) : make_double2(0, 0));
          double2* nx = sl + ((j + 1) & 1) * 17;
          nx[i] = v2;
          if (i == 0) nx[16] = Rf.tau;
          R[(ridx + j + 1) * kNB + i] = i == 0 ? Rf.tau : v2;
        }
      }
      // both warps of the pair are done with this step
      asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");
      if (!ewarp) {
        // column s after its reflector: beta, zeros below (nothing reads it
        // before the tridiagonal is extracted)
        if (j == 0 && lane < len) Bd[(size_t)s * kBandLd + 1 + lane] = lane == 0 ? make_double2(beta, 0) : make_double2(0, 0);
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          st_release_shared(&prog[pair], s * kProgStride + j + 1);
        }
      }
    }
  }
  __syncthreads();
  // tridiagonal T after the reflectors above: d real, e real (beta); the
  // unused e[ld - 1] carries the wait status (1: a wait gave up)
  double* de = reinterpret_cast<double*>(R + ceil_sum(ld - 1) * kNB);
  for (int c = tid; c < ld; c += kS2Thr) {
    de[c] = Bd[(size_t)c * kBandLd].x;
    de[ld + c] = c + 1 < ld ? Bd[(size_t)c * kBandLd + 1].x : (*err ? 1.0 : 0.0);
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
// with the inverse-iteration iterates in shared memory (n * nvec doubles after
// the work arrays), when three CTAs still share an SM
__host__ __device__ inline size_t tri_smem_xbytes(int n, int nval, int nvec) {
  return (tri_smem_bytes(n, nval, nvec) + 7) / 8 * 8 + sizeof(double) * (size_t)n * nvec;
}
constexpr size_t kTriXsmMax = 72 * 1024;

__global__ void __launch_bounds__(kTriThr) tri_eig_kernel(const EigItem* __restrict__ items,
                                                     const double2* __restrict__ rbuf, double* __restrict__ wbuf,
                                                     double2* __restrict__ zbuf, double* __restrict__ scratch,
                                                     int* __restrict__ info, int xsm_ok) {
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
  if (de[2 * ld - 1] != 0.0) {  // the bulge chase gave up a wait: T is incomplete
    if (tid == 0) info[blockIdx.x] = 3;
    return;
  }
  const TriWork tw{d, e, e2, red, lam, lo, hi, xs, cnt, clus, misc};
  const int status = tri_eigvals(tw, n, nval, wbuf + it.w_off, it.bisect_cap);
  double* xsm = xsm_ok ? reinterpret_cast<double*>(smraw + (tri_smem_bytes(n, nval, nvec) + 7) / 8 * 8) : nullptr;
  if (nvec > 0 && status == 0) tri_eigvecs(tw, n, nvec, zbuf + it.z_off, scratch + it.s_off, blockIdx.x, xsm);
  if (tid == 0) info[blockIdx.x] = status;
}

// ----------------------------------------------------------- back-transform
constexpr int kPfSweeps = 4;  // the band reflectors are prefetched into L2 this many sweeps ahead

__host__ __device__ inline size_t back_smem_bytes(int ld, int vb) {
  // Z [ld][vb], one sweep's reflectors [2][ceil(ld/16)][16], W [16][vb], T [16][17]
  return sizeof(double2) * ((size_t)ld * vb + 2 * ((ld + kNB - 1) / kNB) * kNB + kNB * vb + kNB * 17);
}
// reflector entries of a sweep that one thread stages (ceil(kMaxLd / 16) * 16 / 256)
constexpr int kBackStage = (kMaxLd + kThr - 1) / kThr;
// eigenvectors per back-transform CTA: up to kVecBlock, and few enough that
// two CTAs share an SM (the stage is latency-bound) up to ld = 800
inline int back_vec_block(int ld, int max_nvec) {
  int vb = std::min(kVecBlock, std::max(max_nvec, 1));
  // beyond ld = 800 one CTA per SM with more vectors each: every CTA reads all
  // band reflectors (ld^2 / 2 complex) once
  const size_t lim = (size_t)(ld > kVSmemLd ? 200 : 112) * 1024;
  while (vb > 1 && back_smem_bytes(ld, vb) > lim) --vb;
  return vb;
}

// element r of column i of a panel's explicit V (unit diagonal, zeros above;
// below the diagonal the reflectors that stage 1 left in place)
__device__ __forceinline__ double2 panel_v(const double2* __restrict__ vcol, int r, int i) {
  return r > i ? __ldg(vcol + r) : make_double2(r == i ? 1.0 : 0.0, 0.0);
}

// Z (the eigenvectors of T, in shared memory) -> eigenvectors of H. The band
// reflectors of a sweep are prefetched into L2 kPfSweeps sweeps earlier and
// loaded into registers while the previous sweep is applied, then stored to
// shared memory (one barrier per sweep); the panels' reflectors are read
// straight from global memory (the vectors of a CTA all use the same ones,
// so they come from L1 after the first thread).
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
  double2* W = RB + 2 * maxsteps * kNB;            // [16][nv]
  double2* T = W + kNB * nv;                       // [16][17]
  for (int idx = tid; idx < ld * nv; idx += kThr) {
    const int r = idx / nv, k = idx % nv;
    Z[idx] = r < n ? zg[(size_t)(k0 + k) * n + r] : make_double2(0, 0);
  }
  auto prefetch_sweep = [&](int s) {  // one 128-byte line per thread
    const int lines = sweep_steps(ld, s) * kNB * (int)sizeof(double2) / 128;
    if (tid < lines)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(R + sweep_first(ld, s) * kNB + tid * (128 / sizeof(double2))));
  };
  for (int s = ld - 2; s > ld - 2 - kPfSweeps && s >= 0; --s) prefetch_sweep(s);
  auto load_sweep = [&](int s, double2 (&st)[kBackStage]) {
    const int cnt = sweep_steps(ld, s) * kNB;
    const double2* src = R + sweep_first(ld, s) * kNB;
#pragma unroll
    for (int u = 0; u < kBackStage; ++u) {
      const int idx = tid + u * kThr;
      st[u] = idx < cnt ? __ldg(src + idx) : make_double2(0, 0);
    }
  };
  auto store_sweep = [&](double2* dst, const double2 (&st)[kBackStage]) {
#pragma unroll
    for (int u = 0; u < kBackStage; ++u)
      if (tid + u * kThr < maxsteps * kNB) dst[tid + u * kThr] = st[u];
  };
  {
    double2 st[kBackStage];
    load_sweep(ld - 2, st);
    store_sweep(RB, st);
  }
  __syncthreads();
  // ---- band reflectors, sweeps in reverse; one sweep's reflectors act on
  // disjoint rows and are applied together (one thread per reflector and vector)
  for (int s = ld - 2; s >= 0; --s) {
    if (s - kPfSweeps >= 0) prefetch_sweep(s - kPfSweeps);
    double2 st[kBackStage];
    if (s > 0) load_sweep(s - 1, st);  // lands while this sweep is applied
    const int ns = sweep_steps(ld, s);
    const double2* Rs = RB + ((ld - 2 - s) & 1) * maxsteps * kNB;
    for (int task = tid; task < ns * nv; task += kThr) {
      const int j = task / nv, k = task % nv;
      const int p = s + 1 + kNB * j, len = min(kNB, ld - p);
      const double2* v = Rs + j * kNB;
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
    if (s > 0) store_sweep(RB + ((ld - 1 - s) & 1) * maxsteps * kNB, st);
    __syncthreads();
  }
  // ---- panels in reverse: Z[r0:] -= V (T (V^H Z[r0:]))
  for (int c0 = ld - 2 * kNB; c0 >= 0; c0 -= kNB) {
    const int r0 = c0 + kNB, m = ld - r0;
    for (int idx = tid; idx < kNB * kNB; idx += kThr) {
      const int i = idx % kNB, j = idx / kNB;
      T[i * 17 + j] = __ldg(A + (size_t)(r0 + j) * ld + c0 + i);
    }
    // W = V^H Z[r0:]: thread (i, k), two chains over the rows
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      const int idx = tid + o * kThr;
      if (idx < kNB * nv) {
        const int i = idx / nv, k = idx % nv;
        const double2* vcol = A + (size_t)(c0 + i) * ld + r0;
        const double2* zc = Z + (size_t)r0 * nv + k;
        double2 a0 = make_double2(0, 0), a1 = make_double2(0, 0);
        int r = i;  // V is zero above its diagonal
#pragma unroll 4
        for (; r + 1 < m; r += 2) {
          a0 = cadd(a0, cmulc(panel_v(vcol, r, i), zc[(size_t)r * nv]));
          a1 = cadd(a1, cmulc(panel_v(vcol, r + 1, i), zc[(size_t)(r + 1) * nv]));
        }
        if (r < m) a0 = cadd(a0, cmulc(panel_v(vcol, r, i), zc[(size_t)r * nv]));
        W[idx] = cadd(a0, a1);
      }
    }
    __syncthreads();
    // W <- T W (T upper triangular): thread per column k
    for (int k = tid; k < nv; k += kThr) {
      double2 w[kNB];
#pragma unroll
      for (int i = 0; i < kNB; ++i) w[i] = W[i * nv + k];
#pragma unroll
      for (int i = 0; i < kNB; ++i) {
        double2 sacc = make_double2(0, 0);
#pragma unroll
        for (int q = i; q < kNB; ++q) sacc = cadd(sacc, cmul(T[i * 17 + q], w[q]));
        W[i * nv + k] = sacc;
      }
    }
    __syncthreads();
    // Z[r0:] -= V W: thread (row, k)
    for (int idx = tid; idx < m * nv; idx += kThr) {
      const int r = idx / nv, k = idx % nv;
      double2 s0 = make_double2(0, 0), s1 = make_double2(0, 0);
#pragma unroll
      for (int i = 0; i < kNB; i += 2) {
        s0 = cadd(s0, cmul(panel_v(A + (size_t)(c0 + i) * ld + r0, r, i), W[i * nv + k]));
        s1 = cadd(s1, cmul(panel_v(A + (size_t)(c0 + i + 1) * ld + r0, r, i + 1), W[(i + 1) * nv + k]));
      }
      double2* z = Z + (size_t)(r0 + r) * nv + k;
      *z = csub(*z, cadd(s0, s1));
    }
    __syncthreads();
  }
  for (int idx = tid; idx < n * nv; idx += kThr) {
    const int k = idx / n, r = idx % n;
    zg[(size_t)(k0 + k) * n + r] = Z[(size_t)r * nv + k];
  }
}

// ------------------------------------------------------------------- host
int heev2_ld(int n) { return (n + kNB - 1) / kNB * kNB; }

bool heev2_supported(int max_n) { return heev2_ld(max_n) >= 96 && heev2_ld(max_n) <= kMaxLd; }

size_t heev2_rbuf_double2(int ld, int launch_ld) {
  return (size_t)band_off(ld) + (launch_ld > kSmemLd ? (size_t)kBandLd * ld : 0);
}

cudaError_t launch_heev2(const EigItem* items, int nitems, int max_n, int max_nval, int max_nvec, double2* hbuf,
                         double* wbuf, double2* zbuf, double* scratch, double2* rbuf, int* info, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  if (!heev2_supported(max_n)) return cudaErrorInvalidValue;
  const int ld = heev2_ld(max_n);
  cudaError_t e;
  const int mr = sb_rows(ld);
  const bool big = ld > kSmemLd;  // Y and the band in the reflector buffer's work areas
  const size_t s1 = sb_smem_bytes(ld, mr, big, ld > kVSmemLd);
  auto sb = mr == 9    ? sb_kernel<9, false>
            : mr == 17 ? sb_kernel<17, false>
            : mr == 25 ? sb_kernel<25, false>
            : mr == 36 ? sb_kernel<36, true>
            : mr == 49 ? sb_kernel<49, true>
                       : sb_kernel<75, true, true>;
  e = cudaFuncSetAttribute(sb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1);
  if (e != cudaSuccess) return e;
  sb<<<nitems, kThr, s1, st>>>(items, hbuf, rbuf);
  const size_t s2 = sbtrd_smem_bytes(ld, big);
  auto tr = big ? sbtrd_kernel<true> : sbtrd_kernel<false>;
  e = cudaFuncSetAttribute(tr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2);
  if (e != cudaSuccess) return e;
  tr<<<nitems, kS2Thr, s2, st>>>(items, hbuf, rbuf);
  const int xsm_ok = tri_smem_xbytes(max_n, max_nval, max_nvec) <= kTriXsmMax ? 1 : 0;
  const size_t s3 = xsm_ok ? tri_smem_xbytes(max_n, max_nval, max_nvec) : tri_smem_bytes(max_n, max_nval, max_nvec);
  e = cudaFuncSetAttribute(tri_eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s3);
  if (e != cudaSuccess) return e;
  tri_eig_kernel<<<nitems, kTriThr, s3, st>>>(items, rbuf, wbuf, zbuf, scratch, info, xsm_ok);
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
