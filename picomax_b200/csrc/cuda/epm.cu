// Stage 1 kernels: H(k) assembly and the batched FP64 Hermitian eigensolver.
//
// H(k) follows HamiltonianEPM (src/pmx_epm.cpp:56-153): kinetic diagonal
// KCON (2pi/a)^2 |k+G_i|^2, local pseudopotential V(G_i-G_j) off the diagonal,
// and the spin-orbit block i VSO(G_j-G_i) ((k+G_j) x (k+G_i)) . sigma placed
// at (2i, 2j) for j <= i. The reference only fills the lower triangle and its
// eigensolver reads that triangle; here the upper triangle is written as the
// conjugate transpose of the lower one, which is the matrix the reference
// diagonalises.
//
// The eigensolver replaces Eigen::SelfAdjointEigenSolver (called at
// src/pmx_epm.cpp:232, :402, src/pmx_chi.cpp:388, :476). One CTA owns one
// matrix: Householder tridiagonalisation with the rank-2 update of step j-1
// fused into the matrix-vector pass of step j (one read+write of the trailing
// block per step), multisection bisection for the lowest nev eigenvalues,
// inverse iteration with reorthogonalisation inside eigenvalue clusters for
// the tridiagonal eigenvectors, then the back-transform by the stored
// reflectors. Only the eigenpairs the caller needs are formed.
#include <cfloat>
#include <algorithm>
#include <cmath>

#include "pmx_common.cuh"
#include "pmx_device.hpp"
#include "pmx_tri.cuh"
#include "pmx_trieig.cuh"

namespace pmx {
namespace dev {

// ------------------------------------------------------------------ assembly
__global__ void __launch_bounds__(256) assemble_kernel(const CrystalDev* __restrict__ crystals,
                                                       const EigItem* __restrict__ items,
                                                       double2* __restrict__ hbuf) {
  const EigItem it = items[blockIdx.y];
  const CrystalDev C = crystals[it.crystal];
  const int npw = C.npw, n = it.n, side = C.side, off = 2 * C.imax;
  const int ld = it.ld > 0 ? it.ld : n;
  double2* H = hbuf + it.h_off;
  if (ld > n) {  // zero padding: rows n..ld-1 of every column, then columns n..ld-1
    const long long pr = (long long)(ld - n) * ld, total = pr + (long long)n * (ld - n);
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
      if (idx < pr)
        H[(idx / (ld - n)) * ld + n + idx % (ld - n)] = make_double2(0, 0);
      else
        H[(n + (idx - pr) / n) * (long long)ld + (idx - pr) % n] = make_double2(0, 0);
    }
  }
  const double kx = it.k[0], ky = it.k[1], kz = it.k[2];
  const long long total = (long long)npw * npw;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % npw), j = (int)(idx / npw);
    // (a, b) is the lower-triangle block this entry derives from.
    const bool lower = i >= j;
    const int a = lower ? i : j, b = lower ? j : i;
    double2 h0;
    if (a == b) {
      const double gx = kx + C.G[3 * a], gy = ky + C.G[3 * a + 1], gz = kz + C.G[3 * a + 2];
      h0 = make_double2(C.kin * ((gx * gx + gy * gy) + gz * gz), 0.0);
    } else {
      const int dh = C.hkl[3 * a] - C.hkl[3 * b] + off, dk = C.hkl[3 * a + 1] - C.hkl[3 * b + 1] + off,
                dl = C.hkl[3 * a + 2] - C.hkl[3 * b + 2] + off;
      h0 = C.vloc[((long long)dh * side + dk) * side + dl];
    }
    if (!C.soc) {
      H[(long long)j * ld + i] = lower ? h0 : cconj(h0);
      continue;
    }
    // spin-orbit block of the lower pair (a, b): q = G_b - G_a
    double2 blk[2][2];
    blk[0][0] = h0;
    blk[1][1] = h0;
    blk[0][1] = make_double2(0, 0);
    blk[1][0] = make_double2(0, 0);
    if (a != b) {
      const int dh = C.hkl[3 * b] - C.hkl[3 * a] + off, dk = C.hkl[3 * b + 1] - C.hkl[3 * a + 1] + off,
                dl = C.hkl[3 * b + 2] - C.hkl[3 * a + 2] + off;
      const double2 vso = C.vso[((long long)dh * side + dk) * side + dl];
      if (vso.x != 0.0 || vso.y != 0.0) {
        const double ax = kx + C.G[3 * a], ay = ky + C.G[3 * a + 1], az = kz + C.G[3 * a + 2];
        const double bx = kx + C.G[3 * b], by = ky + C.G[3 * b + 1], bz = kz + C.G[3 * b + 2];
        // (k+G_b) x (k+G_a)
        const double cx = by * az - bz * ay, cy = bz * ax - bx * az, cz = bx * ay - by * ax;
        const double2 iv = make_double2(-vso.y, vso.x);  // i * VSO
        const double2 sx = cscale(iv, cx), sy = cscale(iv, cy), sz = cscale(iv, cz);
        blk[0][0] = cadd(blk[0][0], sz);
        blk[1][1] = csub(blk[1][1], sz);
        blk[0][1] = make_double2(sx.x + sy.y, sx.y - sy.x);  // Sx - i Sy
        blk[1][0] = make_double2(sx.x - sy.y, sx.y + sy.x);  // Sx + i Sy
      }
    }
    double2* col0 = H + (long long)(2 * j) * ld + 2 * i;
    double2* col1 = col0 + ld;
    if (lower) {
      col0[0] = blk[0][0];
      col0[1] = blk[1][0];
      col1[0] = blk[0][1];
      col1[1] = blk[1][1];
    } else {  // H[2i+s, 2j+t] = conj(block_(j,i)[t][s])
      col0[0] = cconj(blk[0][0]);
      col0[1] = cconj(blk[0][1]);
      col1[0] = cconj(blk[1][0]);
      col1[1] = cconj(blk[1][1]);
    }
  }
}

cudaError_t launch_assemble(const CrystalDev* crystals, const EigItem* items, int nitems, int max_npw,
                            double2* hbuf, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  long long total = (long long)max_npw * max_npw;
  int bx = (int)((total + 255) / 256);
  if (bx > 512) bx = 512;
  dim3 grid(bx, nitems);
  assemble_kernel<<<grid, 256, 0, st>>>(crystals, items, hbuf);
  return cudaGetLastError();
}

// --------------------------------------------------------------- eigensolver
namespace {

constexpr int kHeevThreads = 256;
constexpr int kWarps = kHeevThreads / 32;
// Lower triangle of an n x n matrix; col(c)[r - c] = A(r, c) for r >= c.
struct LowerFull {  // column-major in global memory, leading dimension ld (upper half unused)
  double2* A;
  int ld;
  __device__ __forceinline__ double2* col(int c) const { return A + (size_t)c * ld + c; }
};
struct LowerPacked {  // packed columns in shared memory
  double2* A;
  int n;
  __device__ __forceinline__ double2* col(int c) const {
    return A + ((size_t)c * n - (size_t)c * (c - 1) / 2);
  }
};

}  // namespace

// Shared-memory layout (double2 unless noted):
//   [packed lower A: n(n+1)/2 if resident] vprev[n] wprev[n] vcur[n] dotp[n] tau[n] part[kWarps*n]
//   doubles: d[n] e[n] e2[n] red[2*kWarps] lam[nev] lo[nev] hi[nev] xs[kHeevThreads]
//   ints: cnt[kHeevThreads] clus[nev+1] misc[4]
// ring = depth of the per-warp prefetch ring of the global-memory path
// (0 = direct loads from L2).
// With MAXS >= kPartGlobalMaxs (n > 832) the per-warp partial sums part[]
// live in the item's global scratch instead (see heev_scratch_doubles).
constexpr int kPartGlobalMaxs = 38;

__host__ __device__ inline size_t heev_smem_bytes(int n, int nev, bool resident, int maxs = 0, int ring = 0) {
  size_t b = 0;
  if (resident) b += (size_t)n * (n + 1) / 2 * sizeof(double2);
  if (!resident && maxs > 0) b += (size_t)kWarps * ring * 32 * maxs * sizeof(double2);
  b += (size_t)(6 + (maxs >= kPartGlobalMaxs ? 0 : kWarps)) * n * sizeof(double2);
  b += (size_t)(3 * n + 2 * kWarps + 3 * nev + kHeevThreads) * sizeof(double);
  b += (size_t)(kHeevThreads + nev + 1 + 4) * sizeof(int);
  return b;
}

// Householder tridiagonalisation (zhetd2 convention, lower triangle only).
// Step j: warp 0 finishes column j (pending rank-2 update of step j-1, then
// the reflector); all warps then make one pass over the trailing lower
// triangle that applies the pending update and accumulates y = A v (rows in
// per-lane registers, column dots by warp reduction) and v^H A v; finally
// w = tau y - tau^2/2 (v^H A v) v becomes the pending update. Three barriers
// per step. MAXS = ceil(n / 32) register slots per lane.
// YS: the per-lane row partials of y accumulate in the warp's row of part[]
// (shared memory) instead of registers, for schedules with more CTAs per SM.
template <int MAXS, int RING, class Acc, bool YS = false>
__device__ __forceinline__ void tridiag_lower(Acc acc, int n, double2* vprev, double2* wprev, double2* vcur,
                                              double2* dotp, double2* tau, double2* part, double2* cnext,
                                              double2* wring, double* d, double* e, double* red) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  bool pending = false;
  bool staged = false;  // column j is in cnext (rows >= j), as left by the previous fused pass
  for (int j = 0; j < n - 1; ++j) {
    // ---- A: column j (warp 0), from shared memory when staged
    if (wid == 0) {
      double2* cj = acc.col(j);
      double xn = 0.0;
      for (int r = j + lane; r < n; r += 32) {
        double2 a = staged ? cnext[r] : cj[r - j];
        if (pending) a = csub(a, cadd(cmul(vprev[r], cconj(wprev[j])), cmul(wprev[r], cconj(vprev[j]))));
        cnext[r] = a;
        if (r >= j + 2) xn += a.x * a.x + a.y * a.y;
      }
      xn = warp_sum(xn);
      __syncwarp();
      const double2 ajj = cnext[j];
      const double2 alpha = cnext[j + 1];
      double beta;
      double2 tj, scal;
      if (xn == 0.0 && alpha.y == 0.0) {
        tj = make_double2(0, 0);
        beta = alpha.x;
        scal = make_double2(1, 0);
      } else {
        beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn), alpha.x);
        tj = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
        const double2 den = make_double2(alpha.x - beta, alpha.y);
        const double dd = den.x * den.x + den.y * den.y;
        scal = make_double2(den.x / dd, -den.y / dd);
      }
      __syncwarp();
      // the reflector v_j stays in column j for the back-transform
      for (int r = j + 2 + lane; r < n; r += 32) {
        const double2 a = cmul(cnext[r], scal);
        cj[r - j] = a;
        vcur[r] = a;
      }
      if (lane == 0) {
        d[j] = ajj.x;
        e[j] = beta;
        tau[j] = tj;
        vcur[j + 1] = make_double2(1, 0);
        cj[1] = make_double2(1, 0);
      }
    }
    __syncthreads();
    const double2 tj = tau[j];
    const bool active = tj.x != 0.0 || tj.y != 0.0;
    // ---- B: fused pass over the trailing lower triangle
    double2 yreg[YS ? 1 : MAXS];
#pragma unroll
    for (int s = 0; s < (YS ? 1 : MAXS); ++s) yreg[s] = make_double2(0, 0);
    if (YS) {
#pragma unroll
      for (int s = 0; s < MAXS; ++s) {
        const int r = 32 * s + lane;
        if (r >= j + 1 && r < n) part[wid * n + r] = make_double2(0, 0);
      }
    }
    double vhav = 0.0;  // the same on every lane
    if (active || pending) {
      // Columns c = c0 + kWarps t of this warp. With RING > 0 every lane
      // prefetches its own rows of the next RING columns into a per-warp ring
      // in shared memory (cp.async); each lane reads back only what it copied,
      // so the per-thread wait_group is the only synchronisation.
      const int c0 = j + 1 + wid;
      double2* ring = wring + (size_t)wid * (RING > 0 ? RING : 1) * 32 * MAXS;
      auto issue = [&](int t) {
        if (RING > 0) {
          const int c = c0 + kWarps * t;
          if (c < n) {
            const double2* cc = acc.col(c);
            double2* buf = ring + (t % (RING > 0 ? RING : 1)) * 32 * MAXS;
#pragma unroll
            for (int s = 0; s < MAXS; ++s) {
              const int r = 32 * s + lane;
              if (r >= c && r < n) cp_async16(buf + 32 * s + lane, cc + (r - c));
            }
          }
          cp_async_commit();
        }
      };
      // rows r >= c of column c (t-th of this warp) into a[]; slots wholly
      // above the diagonal or below the matrix are skipped with warp-uniform
      // branches, not predicated
      auto load = [&](int c, int t, double2 (&a)[MAXS]) {
        if (RING > 0) {
          cp_async_wait<(RING > 0 ? RING - 1 : 0)>();
          const double2* buf = ring + (t % (RING > 0 ? RING : 1)) * 32 * MAXS;
#pragma unroll
          for (int s = 0; s < MAXS; ++s) {
            const int r = 32 * s + lane;
            a[s] = make_double2(0, 0);
            if (32 * s + 31 >= c && 32 * s < n && r >= c && r < n) a[s] = buf[32 * s + lane];
          }
        } else {
          const double2* cc = acc.col(c);
#pragma unroll
          for (int s = 0; s < MAXS; ++s) {
            const int r = 32 * s + lane;
            a[s] = make_double2(0, 0);
            if (32 * s + 31 >= c && 32 * s < n && r >= c && r < n) a[s] = cc[r - c];
          }
        }
      };
      // pending update, store back, row partials of y, this lane's column dot
      auto update = [&](int c, const double2 (&a)[MAXS]) {
        double2* cc = acc.col(c);
        const double2 vc = vcur[c];
        const double2 wcc = cconj(wprev[c]), vcc = cconj(vprev[c]);
        double2 dot = make_double2(0, 0);
#pragma unroll
        for (int s = 0; s < MAXS; ++s) {
          if (32 * s + 31 < c || 32 * s >= n) continue;  // warp-uniform
          const int r = 32 * s + lane;
          if (r >= c && r < n) {
            double2 v = a[s];
            if (pending) {
              v = csub(v, cadd(cmul(vprev[r], wcc), cmul(wprev[r], vcc)));
              if (c == j + 1)
                cnext[r] = v;  // next step's column, kept on chip
              else
                cc[r - c] = v;
            } else if (c == j + 1) {
              cnext[r] = v;
            }
            if (active) {
              if (YS)
                part[wid * n + r] = cadd(part[wid * n + r], cmul(v, vc));
              else
                yreg[YS ? 0 : s] = cadd(yreg[YS ? 0 : s], cmul(v, vc));
              if (r > c) dot = cadd(dot, cmulc(v, vcur[r]));
            }
          }
        }
        return dot;
      };
      auto finish = [&](int c, double2 dot) {
        if (active) {
          dot = warp_sum2(dot);
          if (lane == 0) dotp[c] = dot;
          vhav += cmulc(vcur[c], dot).x;  // conj(v_c) (column part of y_c), same on every lane
        }
      };
#pragma unroll
      for (int t = 0; t < RING; ++t) issue(t);
      for (int t = 0; c0 + kWarps * t < n; ++t) {
        const int c = c0 + kWarps * t;
        double2 a[MAXS];
        load(c, t, a);
        const double2 dot = update(c, a);
        issue(t + RING);
        finish(c, dot);
      }
      if (RING > 0) cp_async_wait<0>();
    }
    if (active) {
      // v^H A v = sum_r conj(v_r) y_r with y = sum over warps of the row
      // partials plus the column dots; this warp's share of both (the column
      // dot share was added once per column above, identically on all lanes).
      double vrow = 0.0;
#pragma unroll
      for (int s = 0; s < MAXS; ++s) {
        const int r = 32 * s + lane;
        if (r >= j + 1 && r < n) {
          if (!YS) part[wid * n + r] = yreg[YS ? 0 : s];
          vrow += cmulc(vcur[r], part[wid * n + r]).x;
        }
      }
      vhav = warp_sum(vrow) + vhav;
      if (lane == 0) red[wid] = vhav;
    }
    __syncthreads();
    // ---- C: w = tau (A v) - |tau|^2/2 (v^H A v) v becomes the pending update
    if (active) {
      double vAv = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) vAv += red[w];
      const double al = -0.5 * (tj.x * tj.x + tj.y * tj.y) * vAv;
      for (int r = j + 1 + tid; r < n; r += kHeevThreads) {
        double2 sum = dotp[r];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sum = cadd(sum, part[w * n + r]);
        const double2 yr = cmul(tj, sum);
        const double2 vr = vcur[r];
        wprev[r] = cadd(yr, cscale(vr, al));
        vprev[r] = vr;
      }
    }
    staged = active || pending;
    pending = active;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double2 a = staged ? cnext[n - 1] : acc.col(n - 1)[0];
    if (pending && n > 1)
      a = csub(a, cadd(cmul(vprev[n - 1], cconj(wprev[n - 1])), cmul(wprev[n - 1], cconj(vprev[n - 1]))));
    d[n - 1] = a.x;
    if (n == 1) tau[0] = make_double2(0, 0);
  }
  __syncthreads();
}

// OCC > 0 overrides the number of resident CTAs per SM the registers are sized
// for; YS keeps the row partials in shared memory (see tridiag_lower).
template <bool RESIDENT, int MAXS, int RING, int OCC = 0, bool YS = false>
__global__ void __launch_bounds__(kHeevThreads, OCC > 0 ? OCC : ((RING >= 2 || MAXS > 9) ? 1 : 2)) heev_kernel(const EigItem* __restrict__ items,
                                                               double2* __restrict__ hbuf,
                                                               double* __restrict__ wbuf,
                                                               double2* __restrict__ zbuf,
                                                               double* __restrict__ scratch,
                                                               int* __restrict__ info,
                                                               double* __restrict__ tri_out) {
  const EigItem it = items[blockIdx.x];
  const int n = it.n, nev = it.nval, nvec = it.want_vec ? it.nev : 0;
  const int ld = it.ld > 0 ? it.ld : n;  // leading dimension of the item's matrix
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nthr = blockDim.x, nw = nthr >> 5;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* sp = reinterpret_cast<double2*>(smraw);
  double2* Apacked = sp;
  if (RESIDENT) sp += (size_t)n * (n + 1) / 2;
  double2* vprev = sp;
  double2* wprev = vprev + n;
  double2* vcur = wprev + n;
  double2* dotp = vcur + n;
  double2* tau = dotp + n;
  constexpr bool kPartG = !RESIDENT && MAXS >= kPartGlobalMaxs;
  double2* part = kPartG ? reinterpret_cast<double2*>(scratch + it.s_off + (size_t)4 * n * (nvec > 0 ? nvec : 1))
                         : tau + n;
  double2* cnext = kPartG ? tau + n : part + (size_t)kWarps * n;
  double2* wring = cnext + n;  // per-warp prefetch ring (global-memory path)
  if (!RESIDENT) sp = wring + (size_t)kWarps * RING * 32 * MAXS;
  else sp = wring;
  double* d = reinterpret_cast<double*>(sp);
  double* e = d + n;
  double* e2 = e + n;
  double* red = e2 + n;
  double* lam = red + 2 * kWarps;
  double* lo = lam + nev;
  double* hi = lo + nev;
  double* xs = hi + nev;
  int* cnt = reinterpret_cast<int*>(xs + kHeevThreads);
  int* clus = cnt + kHeevThreads;
  int* misc = clus + nev + 1;

  const double2* src = hbuf + it.h_off;
  if (RESIDENT) {
    const LowerPacked pk{Apacked, n};
    for (int c = wid; c < n; c += nw) {
      double2* dst = pk.col(c);
      for (int r = c + lane; r < n; r += 32) dst[r - c] = src[(size_t)c * ld + r];
    }
    __syncthreads();
    tridiag_lower<MAXS, 0>(pk, n, vprev, wprev, vcur, dotp, tau, part, cnext, wring, d, e, red);
  } else {
    tridiag_lower<MAXS, RING, LowerFull, YS>(LowerFull{hbuf + it.h_off, ld}, n, vprev, wprev, vcur, dotp, tau, part,
                                             cnext, wring,
                              d, e, red);
  }

  // ------------------------------------------------------------- eigenvalues
  const TriWork tw{d, e, e2, red, lam, lo, hi, xs, cnt, clus, misc};
  const int status = tri_eigvals(tw, n, nev, wbuf + it.w_off, it.bisect_cap);
  if (tri_out) {
    // H = Q T Q^H for the adjoint: T (d, e after deflation), the reflector
    // scalars tau, and (resident path) the reflectors back into hbuf
    double* t = tri_out + (size_t)blockIdx.x * 4 * n;
    for (int i = tid; i < n; i += nthr) {
      t[i] = d[i];
      t[n + i] = i < n - 1 ? e[i] : 0.0;
      t[2 * n + 2 * i] = tau[i].x;
      t[2 * n + 2 * i + 1] = i < n - 1 ? tau[i].y : 0.0;
      if (i == n - 1) t[2 * n + 2 * i] = 0.0;
    }
    if (RESIDENT) {
      const LowerPacked pk{Apacked, n};
      double2* dst = hbuf + it.h_off;
      for (int c = wid; c < n; c += nw) {
        const double2* col = pk.col(c);
        for (int r = c + lane; r < n; r += 32) dst[(size_t)c * ld + r] = col[r - c];
      }
    }
  }
  if (!it.want_vec || status != 0) {
    if (tid == 0) info[blockIdx.x] = status;
    return;
  }

  // ----------------------------------------------- tridiagonal eigenvectors
  tri_eigvecs(tw, n, nvec, zbuf + it.z_off, scratch + it.s_off, blockIdx.x);

  // ----------------------------------------------------------- back-transform
  // x = H_0 H_1 ... H_{n-2} z ; one warp per eigenvector, no block barriers.
  if constexpr (!kPartG) {
    // z in this warp's row of part[] (free after the reduction); the reflector
    // v_j is read once per step into registers (slot q: row j + 1 + lane + 32 q),
    // and where the registers allow, v_{j-1} is loaded while v_j is applied.
    constexpr int kOcc = OCC > 0 ? OCC : ((RING >= 2 || MAXS > 9) ? 1 : 2);
    constexpr int kRegs = 65536 / (kHeevThreads * kOcc) < 255 ? 65536 / (kHeevThreads * kOcc) : 255;
    constexpr bool kPf = 8 * MAXS + 48 <= kRegs;
    double2* zs = part + (size_t)wid * n;
    auto vcol = [&](int j) {
      return RESIDENT ? LowerPacked{Apacked, n}.col(j) : LowerFull{hbuf + it.h_off, ld}.col(j);
    };
    for (int k = wid; k < nvec; k += nw) {
      double2* zg = zbuf + it.z_off + (size_t)k * n;
      for (int r = lane; r < n; r += 32) zs[r] = zg[r];
      __syncwarp();
      double2 vr[MAXS], vn[kPf ? MAXS : 1];
#pragma unroll
      for (int q = 0; q < MAXS; ++q) {
        const int r = n - 1 + lane + 32 * q;  // column j = n - 2 (none for n = 1)
        vr[q] = make_double2(0, 0);
        if (n >= 2 && n - 1 + 32 * q < n && r < n) vr[q] = vcol(n - 2)[r - (n - 2)];
      }
      for (int j = n - 2; j >= 0; --j) {
        if (kPf && j > 0) {
          const double2* vp = vcol(j - 1);
#pragma unroll
          for (int q = 0; q < (kPf ? MAXS : 1); ++q) {
            const int r = j + lane + 32 * q;
            vn[q] = make_double2(0, 0);
            if (j + 32 * q < n && r < n) vn[q] = vp[r - (j - 1)];
          }
        }
        const double2 tj = tau[j];
        if (tj.x != 0.0 || tj.y != 0.0) {
          double2 sacc = make_double2(0, 0);
#pragma unroll
          for (int q = 0; q < MAXS; ++q) {
            const int r = j + 1 + lane + 32 * q;
            if (j + 1 + 32 * q < n && r < n) sacc = cadd(sacc, cmulc(vr[q], zs[r]));
          }
          sacc = cmul(tj, warp_sum2(sacc));
#pragma unroll
          for (int q = 0; q < MAXS; ++q) {
            const int r = j + 1 + lane + 32 * q;
            if (j + 1 + 32 * q < n && r < n) zs[r] = csub(zs[r], cmul(vr[q], sacc));
          }
        }
        if (j > 0) {
          if (kPf) {
#pragma unroll
            for (int q = 0; q < MAXS; ++q) vr[q] = vn[kPf ? q : 0];
          } else {
            const double2* vp = vcol(j - 1);
#pragma unroll
            for (int q = 0; q < MAXS; ++q) {
              const int r = j + lane + 32 * q;
              vr[q] = make_double2(0, 0);
              if (j + 32 * q < n && r < n) vr[q] = vp[r - (j - 1)];
            }
          }
        }
      }
      __syncwarp();
      for (int r = lane; r < n; r += 32) zg[r] = zs[r];
      __syncwarp();
    }
  } else {
    for (int k = wid; k < nvec; k += nw) {
      double2* z = zbuf + it.z_off + (size_t)k * n;
      for (int j = n - 2; j >= 0; --j) {
        const double2 tj = tau[j];
        if (tj.x == 0.0 && tj.y == 0.0) continue;
        const double2* v = (RESIDENT ? LowerPacked{Apacked, n}.col(j) : LowerFull{hbuf + it.h_off, ld}.col(j)) - j;
        double2 s = make_double2(0, 0);
        for (int r = j + 1 + lane; r < n; r += 32) s = cadd(s, cmulc(v[r], z[r]));
        s = cmul(tj, warp_sum2(s));
        for (int r = j + 1 + lane; r < n; r += 32) z[r] = csub(z[r], cmul(v[r], s));
        __syncwarp();
      }
    }
  }
  if (tid == 0) info[blockIdx.x] = 0;
}

size_t heev_scratch_doubles(int n, int nvec, int max_n) {
  const int slots = (max_n + 31) / 32;
  return (size_t)4 * n * (nvec > 0 ? nvec : 1) + (slots > 26 ? (size_t)2 * kWarps * n : 0);
}

bool heev_resident(int n, int nev) { return heev_smem_bytes(n, nev, true) <= (size_t)227 * 1024; }

int heev_smem_max_n() {
  // largest n whose resident (packed lower) layout fits the 227 KB opt-in limit
  const size_t lim = 227 * 1024;
  int n = 1;
  while (heev_smem_bytes(n + 1, 64, true) <= lim) ++n;
  return n;
}

namespace {
template <bool RES, int MAXS, int RING, int OCC = 0, bool YS = false>
cudaError_t heev_launch_t(const EigItem* items, int nitems, size_t smem, double2* hbuf, double* wbuf,
                          double2* zbuf, double* scratch, int* info, cudaStream_t st, double* tri, int* occ) {
  cudaError_t err = cudaFuncSetAttribute(heev_kernel<RES, MAXS, RING, OCC, YS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  if (occ)  // resident CTAs per SM instead of a launch
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, heev_kernel<RES, MAXS, RING, OCC, YS>, kHeevThreads,
                                                         smem);
  heev_kernel<RES, MAXS, RING, OCC, YS><<<nitems, kHeevThreads, smem, st>>>(items, hbuf, wbuf, zbuf, scratch,
                                                                                 info, tri);
  return cudaGetLastError();
}
}  // namespace

namespace {
// register slots per lane (template MAXS) for ceil(n / 32) slots; 0 beyond n = 1216
int heev_slot_class(int slots) {
  const int cls[] = {2, 4, 6, 9, 13, 19, 26, 38};
  for (int c : cls)
    if (slots <= c) return c;
  return 0;
}

// One schedule of the global-memory path: prefetch ring depth, row partials in
// shared memory (YS).
struct HeevSched {
  int ring;
  bool ys;
};

// The schedules a matrix size allows, in autotuner order: 0 direct loads,
// then (n <= 416) the prefetch rings whose shared memory fits (one-column,
// three-column) and the row partials in shared memory with one CTA more per SM.
int heev_schedules(int max_n, int max_nev, HeevSched* out) {
  const int slots = (max_n + 31) / 32;
  int k = 0;
  out[k++] = {0, false};
  if (max_n <= heev_smem_max_n() && heev_resident(max_n, max_nev)) return k;  // resident: one schedule
  const int maxs = heev_slot_class(slots);
  const size_t lim = 227 * 1024;
  if (maxs <= 13) {
    if (heev_smem_bytes(max_n, max_nev, false, maxs, 1) <= lim) out[k++] = {1, false};
    if (heev_smem_bytes(max_n, max_nev, false, maxs, 3) <= lim) out[k++] = {3, false};
    const int ctas = maxs <= 9 ? 3 : 2;
    if ((size_t)ctas * (heev_smem_bytes(max_n, max_nev, false, maxs, 0) + 1024) <= (size_t)228 * 1024)
      out[k++] = {0, true};
  }
  return k;
}

template <int S>
cudaError_t heev_dispatch(bool resident, const HeevSched& sc, const EigItem* items, int nitems, size_t smem,
                          double2* hbuf, double* wbuf, double2* zbuf, double* scratch, int* info, cudaStream_t st,
                          double* tri, int* occ) {
  if (resident)
    return heev_launch_t<true, S, 0>(items, nitems, smem, hbuf, wbuf, zbuf, scratch, info, st, tri, occ);
  if constexpr (S <= 13) {
    if (sc.ring == 3)
      return heev_launch_t<false, S, 3>(items, nitems, smem, hbuf, wbuf, zbuf, scratch, info, st, tri, occ);
    if (sc.ring == 1)
      return heev_launch_t<false, S, 1>(items, nitems, smem, hbuf, wbuf, zbuf, scratch, info, st, tri, occ);
    if (sc.ys)
      return heev_launch_t<false, S, 0, (S <= 9 ? 3 : 2), true>(items, nitems, smem, hbuf, wbuf, zbuf, scratch, info,
                                                                st, tri, occ);
  }
  return heev_launch_t<false, S, 0>(items, nitems, smem, hbuf, wbuf, zbuf, scratch, info, st, tri, occ);
}

// Launch (occ == nullptr) or occupancy query of one schedule.
cudaError_t heev_run(const EigItem* items, int nitems, int max_n, int max_nev, double2* hbuf, double* wbuf,
                     double2* zbuf, double* scratch, int* info, cudaStream_t st, int variant, double* tri,
                     int* occ);
}  // namespace

int heev_variants(int max_n, int max_nev) {
  HeevSched sc[8];
  return heev_schedules(max_n, max_nev, sc);
}

cudaError_t launch_heev(const EigItem* items, int nitems, int max_n, int max_nev, double2* hbuf,
                        double* wbuf, double2* zbuf, double* scratch, int* info, cudaStream_t st, int variant,
                        double* tri) {
  if (nitems <= 0) return cudaSuccess;
  return heev_run(items, nitems, max_n, max_nev, hbuf, wbuf, zbuf, scratch, info, st, variant, tri, nullptr);
}

int heev_batch_unit(int max_n, int max_nev) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    return 1;
  int l = 1;
  const int nv = heev_variants(max_n, max_nev);
  for (int v = 0; v < nv; ++v) {
    int occ = 0;
    if (heev_run(nullptr, 0, max_n, max_nev, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, v, nullptr,
                 &occ) != cudaSuccess ||
        occ <= 0)
      continue;
    int a = l, b = occ;
    while (b) {
      const int t = a % b;
      a = b;
      b = t;
    }
    l = l / a * occ;
  }
  return l * sms;
}

namespace {
cudaError_t heev_run(const EigItem* items, int nitems, int max_n, int max_nev, double2* hbuf, double* wbuf,
                     double2* zbuf, double* scratch, int* info, cudaStream_t st, int variant, double* tri,
                     int* occ) {
  const bool resident = max_n <= heev_smem_max_n() && heev_resident(max_n, max_nev);
  const int slots = (max_n + 31) / 32;
  // global-memory path schedules (heev_schedules): direct L2 loads (2 CTAs/SM),
  // one-column prefetch buffer per warp (2 CTAs/SM), three-column ring (1 CTA/SM),
  // direct with the row partials in shared memory and one CTA more per SM.
  // Measured on n = 274 (B200): 82 / 95 / 108 ms per 1787 matrices; a
  // one-CTA-per-SM padding of schedule 0 (L2-resident trailing blocks), a
  // register cap for 3 CTAs/SM and a two-columns-per-iteration pass were
  // slower still (120 / 106 / 97 ms): the pass is bound by dependent FP64
  // chains and load latency at 16 warps per SM. For n = 401 (one CTA per SM by
  // registers) a register cap for two CTAs per SM was slower too (159 vs 141 ms),
  // while the row partials in shared memory at two CTAs per SM are faster:
  // eigenvalues of 778 matrices, n = 401: 115 -> 83 ms (1787 matrices of
  // n = 362: 108 -> 80 ms); at n = 274 and three CTAs per SM 71 vs 68 ms.
  // Two further forms were slower on every size: the column dots of four
  // columns reduced in one transposed butterfly (n = 274 / 401: 75 / 113 ms
  // against 68 / 115), and two columns per warp iteration with the partials
  // in shared memory (83 / 150 ms against 65 / 87).
  HeevSched sc[8];
  const int nsc = heev_schedules(max_n, max_nev, sc);
  const HeevSched sched = sc[std::min(std::max(variant, 0), nsc - 1)];
  const size_t smem = heev_smem_bytes(max_n, max_nev, resident, resident ? 0 : heev_slot_class(slots),
                                      resident ? 0 : sched.ring);
  switch (heev_slot_class(slots)) {
#define PMX_HEEV_CASE(S) \
  case S:                \
    return heev_dispatch<S>(resident, sched, items, nitems, smem, hbuf, wbuf, zbuf, scratch, info, st, tri, occ);
    PMX_HEEV_CASE(2)
    PMX_HEEV_CASE(4)
    PMX_HEEV_CASE(6)
    PMX_HEEV_CASE(9)
    PMX_HEEV_CASE(13)
    PMX_HEEV_CASE(19)
    PMX_HEEV_CASE(26)
    PMX_HEEV_CASE(38)
#undef PMX_HEEV_CASE
    default: return cudaErrorInvalidValue;  // n > 1216
  }
}
}  // namespace

}  // namespace dev
}  // namespace pmx
