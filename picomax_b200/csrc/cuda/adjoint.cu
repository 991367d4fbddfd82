// Adjoint kernels of the band and chi_LL -> eps_M stages (FP64). The forward
// formulas they differentiate are those of chi.cu / epm.cu:
//   O_mn(t)  = M_m(t) conj(M_n(t)),  M_m = sum_p sum_s conj(c_s(p)) v_s(loci[m][p])
//   s_im     = sum_t w_t Re O delta(dE_t - w),  s_re = -sum_t w_t Im O delta(dE_t - w)
//   chi_LL   = pi f1 s + 2 f2 s_pv (kk = 0),  then Kramers-Kronig (kk = 1)
//   eps_mn   = delta_mn + chi_mn (Hermitian fill), eps_M = 1 / [eps^-1]_00
// (src/pmx_chi_copy.cpp:500-615, src/pmx_chi.cpp:272-309,
// include/matlab_wrapper/+picomax/+eps/macroscopic.m:13-29).
#include <cuda_runtime.h>

#include <algorithm>

#include <cfloat>

#include "pmx_adjoint.hpp"
#include "pmx_common.cuh"
#include "pmx_tri.cuh"

namespace pmx {
namespace dev {

namespace {
constexpr double kPiD = 3.14159265358979323846;

__device__ __forceinline__ double2 cconj2(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ void pair_mn(int p, int& m, int& n) {
  m = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
  while ((m + 1) * (m + 2) / 2 <= p) ++m;
  while (m * (m + 1) / 2 > p) --m;
  n = p - m * (m + 1) / 2;
}

// broadening (as chi.cu) and its derivative in x
__device__ __forceinline__ double broaden_d(int model, double eps, double x) {
  switch (model) {
    case 0:
      return exp(-0.5 * x * x / (eps * eps)) / (eps * sqrt(2.0 * kPiD));
    case 1:
      return eps / kPiD / (eps * eps + x * x);
    case 2:
      return fabs(x) < 0.5 * eps ? 4.0 / eps * (0.5 - fabs(x) / eps) : 0.0;
    default:
      return fabs(x) < 0.5 * eps ? 1.0 / eps : 0.0;
  }
}
__device__ __forceinline__ double dbroaden_d(int model, double eps, double x, double d) {
  switch (model) {
    case 0:
      return -x / (eps * eps) * d;
    case 1: {
      const double den = eps * eps + x * x;
      return -2.0 * x * eps / (kPiD * den * den);
    }
    case 2:
      return fabs(x) < 0.5 * eps ? (x > 0 ? -4.0 / (eps * eps) : (x < 0 ? 4.0 / (eps * eps) : 0.0)) : 0.0;
    default:
      return 0.0;
  }
}
}  // namespace

// ------------------------------------------------------------------ eps_M
// One warp per (q, w): Gauss-Jordan inverse of eps with partial pivoting in
// shared memory, then dL/deps_ab = g conj(eps_M^2 B_0a B_b0), folded onto
// the stored n <= m pairs through the Hermitian fill.
__global__ void __launch_bounds__(128) epsm_vjp_kernel(const double* __restrict__ re, const double* __restrict__ im,
                                                       const double2* __restrict__ g, int neps, int nq, int nf,
                                                       double* __restrict__ gre, double* __restrict__ gim) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int job = blockIdx.x * (blockDim.x >> 5) + w;
  if (job >= nq * nf) return;
  const int q = job / nf, f = job % nf;
  const int n = neps, ld = 2 * n;
  double2* E = reinterpret_cast<double2*>(smraw) + (size_t)w * n * ld;
  const int np = n * (n + 1) / 2;
  for (int idx = lane; idx < n * n; idx += 32) {
    const int r = idx / n, c = idx % n;
    const int m = r > c ? r : c, nn = r > c ? c : r;
    const size_t o = ((size_t)q * np + (size_t)m * (m + 1) / 2 + nn) * nf + f;
    double2 v = make_double2(re[o], im[o]);
    if (r < c) v.y = -v.y;
    if (r == c) v.x += 1.0;
    E[r * ld + c] = v;
    E[r * ld + n + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  __syncwarp();
  for (int k = 0; k < n; ++k) {
    double best = -1.0;
    int bi = k;
    for (int r = k + lane; r < n; r += 32) {
      const double2 v = E[r * ld + k];
      const double a = v.x * v.x + v.y * v.y;
      if (a > best) {
        best = a;
        bi = r;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (bi != k)
      for (int c = lane; c < ld; c += 32) {
        const double2 t = E[k * ld + c];
        E[k * ld + c] = E[bi * ld + c];
        E[bi * ld + c] = t;
      }
    __syncwarp();
    const double2 p = E[k * ld + k];
    const double pd = p.x * p.x + p.y * p.y;
    const double2 inv = make_double2(p.x / pd, -p.y / pd);
    __syncwarp();
    for (int c = k + lane; c < ld; c += 32) E[k * ld + c] = cmul(E[k * ld + c], inv);
    __syncwarp();
    for (int r = 0; r < n; ++r) {
      if (r == k) continue;
      const double2 fct = E[r * ld + k];
      __syncwarp();
      for (int c = k + 1 + lane; c < ld; c += 32) E[r * ld + c] = csub(E[r * ld + c], cmul(fct, E[k * ld + c]));
      if (lane == 0) E[r * ld + k] = make_double2(0.0, 0.0);
      __syncwarp();
    }
  }
  // B = eps^-1 = right half; eps_M = 1 / B_00
  const double2 b00 = E[n];
  const double bb = b00.x * b00.x + b00.y * b00.y;
  const double2 em = make_double2(b00.x / bb, -b00.y / bb);
  const double2 em2 = cmul(em, em);
  const double2 gg = g[(size_t)q * nf + f];
  // Ebar_ab = g conj(em2 B_0a B_b0)
  auto ebar = [&](int a, int b) {
    const double2 t = cmul(em2, cmul(E[n + a], E[b * ld + n]));
    return cmul(gg, cconj2(t));
  };
  for (int pp = lane; pp < np; pp += 32) {
    int m, nn;
    pair_mn(pp, m, nn);
    double2 x = ebar(m, nn);
    if (m != nn) x = cadd(x, cconj2(ebar(nn, m)));
    const size_t o = ((size_t)q * np + pp) * nf + f;
    gre[o] = x.x;
    gim[o] = x.y;
  }
}

cudaError_t launch_epsm_vjp(const double* re, const double* im, const double2* g, int neps, int nq, int nf,
                            double* gre, double* gim, cudaStream_t st) {
  if (neps > 64 || neps < 1) return cudaErrorInvalidValue;
  if (nq * nf <= 0) return cudaSuccess;
  const size_t per = (size_t)neps * 2 * neps * sizeof(double2);
  int warps = (int)std::max<size_t>(1, std::min<size_t>(4, (size_t)(200 * 1024) / per));
  const size_t smem = (size_t)warps * per;
  cudaError_t e = cudaFuncSetAttribute(epsm_vjp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int jobs = nq * nf;
  epsm_vjp_kernel<<<(jobs + warps - 1) / warps, 32 * warps, smem, st>>>(re, im, g, neps, nq, nf, gre, gim);
  return cudaGetLastError();
}

// ---------------------------------------------------- Kramers-Kronig transpose
// K[f][s] = w_s / (w_s^2 - w_f^2), s != f; out_s = g_s + ds sum_f K[f][s] h_f
// with h the other half.
__global__ void kk_t_kernel(const double* __restrict__ g, double* __restrict__ out, int rows, int nf,
                            double dfreq) {
  const long long total = 2LL * rows * nf;
  const double ds = dfreq * 2.0 / kPiD;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(idx % nf);
    const long long r = idx / nf;  // [0, 2 rows)
    const long long other = r < rows ? r + rows : r - rows;
    const double* h = g + other * nf;
    const double ws = dfreq * s;
    double acc = 0.0;
    for (int f = 0; f < nf; ++f) {
      if (f == s) continue;
      const double wf = dfreq * f;
      acc += ws / (ws * ws - wf * wf) * h[f];
    }
    out[idx] = g[idx] + ds * acc;
  }
}

cudaError_t launch_kk_t(const double* g, double* out, int rows, int nf, double dfreq, cudaStream_t st) {
  const long long total = 2LL * rows * nf;
  if (total <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  kk_t_kernel<<<blocks, 256, 0, st>>>(g, out, rows, nf, dfreq);
  return cudaGetLastError();
}

// ------------------------------------------------------------- contraction
namespace {
constexpr int kTB = 32, kPB = 32, kFT = 16;
}

__global__ void __launch_bounds__(256) contract_vjp_kernel(ContractVjpArgs a) {
  __shared__ double dl[kTB][kFT + 1], ddl[kTB][kFT + 1];
  __shared__ double gI[kPB][kFT + 1], gR[kPB][kFT + 1];
  __shared__ double pg[kTB][kFT + 1], pgd[kTB][kFT + 1];
  __shared__ double pR[kPB][kFT + 1], pI[kPB][kFT + 1];
  __shared__ double red[8][kTB];
  const int tid = threadIdx.x, tl = tid & 31, pgi = tid >> 5;
  const int t0 = blockIdx.x * kTB, p0 = blockIdx.y * kPB;
  const bool pv = a.f2 != nullptr;
  double acc[4][8];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[j][q] = 0.0;
  for (int f0 = 0; f0 < a.nf; f0 += kFT) {
    for (int idx = tid; idx < kTB * kFT; idx += 256) {
      const int tt = idx / kFT, ff = idx % kFT;
      const int t = t0 + tt, f = f0 + ff;
      double d = 0.0, dd = 0.0, g = 0.0, gd = 0.0;
      if (t < a.T && f < a.nf) {
        const double de = a.dE[t], w = a.dfreq * f;
        const double x = de - w;
        d = broaden_d(a.delta, a.eps, x);
        dd = dbroaden_d(a.delta, a.eps, x, d);
        if (pv) {
          const double den = de * de - w * w;
          g = de / den;
          gd = -(de * de + w * w) / (den * den);
        }
      }
      dl[tt][ff] = d;
      ddl[tt][ff] = dd;
      pg[tt][ff] = g;
      pgd[tt][ff] = gd;
      const int pp = p0 + tt;  // kPB == kTB
      double gi = 0.0, gr = 0.0, pr = 0.0, pi_ = 0.0;
      if (pp < a.np && f < a.nf) {
        const size_t o = (size_t)pp * a.nf + f;
        if (f >= 1) {
          gi = a.f1[pp] * a.gim[o];
          gr = a.f1[pp] * a.gre[o];
        }
        if (pv) {
          pr = a.f2[pp] * a.gre[o];
          pi_ = a.f2[pp] * a.gim[o];
        }
      }
      gI[tt][ff] = gi;
      gR[tt][ff] = gr;
      pR[tt][ff] = pr;
      pI[tt][ff] = pi_;
    }
    __syncthreads();
#pragma unroll 4
    for (int ff = 0; ff < kFT; ++ff) {
      const double d = dl[tl][ff], dd = ddl[tl][ff];
      const double g = pg[tl][ff], gd = pgd[tl][ff];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int pl = pgi + 8 * j;
        const double gi = gI[pl][ff], gr = gR[pl][ff];
        acc[j][0] = fma(gi, d, acc[j][0]);
        acc[j][1] = fma(gr, d, acc[j][1]);
        acc[j][2] = fma(gi, dd, acc[j][2]);
        acc[j][3] = fma(gr, dd, acc[j][3]);
        if (pv) {
          const double pr = pR[pl][ff], pi_ = pI[pl][ff];
          acc[j][4] = fma(pr, g, acc[j][4]);
          acc[j][5] = fma(pi_, g, acc[j][5]);
          acc[j][6] = fma(pr, gd, acc[j][6]);
          acc[j][7] = fma(pi_, gd, acc[j][7]);
        }
      }
    }
    __syncthreads();
  }
  const int t = t0 + tl;
  double dsum = 0.0;
  if (t < a.T) {
    const double kw = a.wgt[t];
    const int A = 3 * a.neps;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int p = p0 + pgi + 8 * j;
      if (p >= a.np) continue;
      int m, n;
      pair_mn(p, m, n);
      const double2 Mm = a.M[(size_t)t * A + 3 * m], Mn = a.M[(size_t)t * A + 3 * n];
      const double2 O = cmulc(Mn, Mm);  // M_m conj(M_n)
      double2 ob = make_double2(kw * (acc[j][0] + acc[j][4]), kw * (-acc[j][1] + acc[j][5]));
      a.obar[(size_t)t * a.np + p] = ob;
      dsum += kw * (O.x * (acc[j][2] + acc[j][6]) + O.y * (-acc[j][3] + acc[j][7]));
    }
  }
  red[pgi][tl] = dsum;
  __syncthreads();
  if (tid < kTB) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) s += red[w][tid];
    const int tt = t0 + tid;
    if (tt < a.T) atomicAdd(a.dEbar + tt, s);
  }
}

cudaError_t launch_contract_vjp(const ContractVjpArgs& a, cudaStream_t st) {
  if (a.T <= 0 || a.np <= 0) return cudaSuccess;
  dim3 grid((a.T + kTB - 1) / kTB, (a.np + kPB - 1) / kPB);
  contract_vjp_kernel<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

__global__ void mbar_kernel(const double2* __restrict__ M, const double2* __restrict__ obar, int T, int neps,
                            double2* __restrict__ mbar) {
  const long long total = (long long)T * neps;
  const int A = 3 * neps, np = neps * (neps + 1) / 2;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long t = idx / neps;
    const int m = (int)(idx % neps);
    const double2* Mt = M + (size_t)t * A;
    const double2* ob = obar + (size_t)t * np;
    double2 s = make_double2(0, 0);
    for (int n = 0; n <= m; ++n) s = cadd(s, cmul(ob[m * (m + 1) / 2 + n], Mt[3 * n]));
    for (int n = m; n < neps; ++n) s = cadd(s, cmul(cconj2(ob[n * (n + 1) / 2 + m]), Mt[3 * n]));
    mbar[idx] = s;
  }
}

cudaError_t launch_mbar(const double2* M, const double2* obar, int T, int neps, double2* mbar, cudaStream_t st) {
  const long long total = (long long)T * neps;
  if (total <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  mbar_kernel<<<blocks, 256, 0, st>>>(M, obar, T, neps, mbar);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- overlaps
// Block (k, y): y < ncd_max -> conduction state y at k, else valence state
// y - ncd_max at k+q. Threads run over the eigenvector components.
__global__ void __launch_bounds__(256) zbar_kernel(ZbarArgs a) {
  const int k = blockIdx.x, y = blockIdx.y;
  const int ncd = a.ncd[k], nvd = a.nvd[k];
  const int n = a.n, npw = a.npw, sw = a.soc ? 2 : 1;
  const long long bo = a.blkoff[k];
  if (y < a.ncd_max) {
    const int c = y;
    if (c >= ncd) return;
    const int stc = a.cidx[a.cbase[k] + c];
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const int s = a.soc ? (r & 1) : 0, p = a.soc ? (r >> 1) : r;
      double2 acc = make_double2(0, 0);
      for (int v = 0; v < nvd; ++v) {
        const long long t = a.dest[bo + (long long)c * nvd + v];
        if (t < 0) continue;
        const double2* vv = a.zq + ((size_t)k * a.nev + a.vidx[a.vbase[k] + v]) * n;
        const double2* mb = a.mbar + (size_t)t * a.neps;
        for (int m = 0; m < a.neps; ++m) {
          const int lp = a.loci[(size_t)m * npw + p];
          if (lp < 0) continue;
          acc = cadd(acc, cmulc(mb[m], vv[sw * lp + s]));  // conj(mbar) v
        }
      }
      a.zbar_k[((size_t)k * a.ns + stc) * n + r] = acc;
    }
    if (threadIdx.x == 0) {
      double l = 0.0;
      for (int v = 0; v < nvd; ++v) {
        const long long t = a.dest[bo + (long long)c * nvd + v];
        if (t >= 0) l += a.dEbar[t];
      }
      a.lbar_k[(size_t)k * a.ns + stc] = l;
    }
  } else {
    const int v = y - a.ncd_max;
    if (v >= nvd) return;
    const int stv = a.vidx[a.vbase[k] + v];
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const int s = a.soc ? (r & 1) : 0, rr = a.soc ? (r >> 1) : r;
      double2 acc = make_double2(0, 0);
      for (int c = 0; c < ncd; ++c) {
        const long long t = a.dest[bo + (long long)c * nvd + v];
        if (t < 0) continue;
        const double2* cv = a.zk + ((size_t)k * a.nev + a.cidx[a.cbase[k] + c]) * n;
        const double2* mb = a.mbar + (size_t)t * a.neps;
        for (int m = 0; m < a.neps; ++m) {
          const int p = a.linv[(size_t)m * npw + rr];
          if (p < 0) continue;
          acc = cadd(acc, cmul(mb[m], cv[sw * p + s]));  // mbar c
        }
      }
      a.zbar_q[((size_t)k * a.ns + stv) * n + r] = acc;
    }
    if (threadIdx.x == 0) {
      double l = 0.0;
      for (int c = 0; c < ncd; ++c) {
        const long long t = a.dest[bo + (long long)c * nvd + v];
        if (t >= 0) l -= a.dEbar[t];
      }
      a.lbar_q[(size_t)k * a.ns + stv] = l;
    }
  }
}

cudaError_t launch_zbar(const ZbarArgs& a, cudaStream_t st) {
  if (a.nk <= 0 || a.ncd_max + a.nvd_max <= 0) return cudaSuccess;
  dim3 grid(a.nk, a.ncd_max + a.nvd_max);
  zbar_kernel<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

// ------------------------------------------------------------ batched ZGEMM
namespace {
constexpr int kGT = 32, kGK = 16;
}

__global__ void __launch_bounds__(256) zgemm_kernel(int conj_a, int M, int N, int K, const double2* __restrict__ A,
                                                    int lda, long long sa, const double2* __restrict__ B, int ldb,
                                                    long long sb, double2* __restrict__ C, int ldc, long long sc) {
  __shared__ double2 As[kGK][kGT + 1];
  __shared__ double2 Bs[kGK][kGT + 1];
  const int b = blockIdx.z;
  A += (size_t)b * sa;
  B += (size_t)b * sb;
  C += (size_t)b * sc;
  const int i0 = blockIdx.x * kGT, j0 = blockIdx.y * kGT;
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  double2 acc[2][2];
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y) acc[x][y] = make_double2(0, 0);
  for (int k0 = 0; k0 < K; k0 += kGK) {
    for (int idx = tid; idx < kGK * kGT; idx += 256) {
      int kk, ii;
      double2 v = make_double2(0, 0);
      if (conj_a) {
        ii = idx / kGK;
        kk = idx % kGK;
        const int i = i0 + ii, k = k0 + kk;
        if (i < M && k < K) v = cconj2(A[(size_t)i * lda + k]);
      } else {
        kk = idx / kGT;
        ii = idx % kGT;
        const int i = i0 + ii, k = k0 + kk;
        if (i < M && k < K) v = A[(size_t)k * lda + i];
      }
      As[kk][ii] = v;
      const int jj = idx / kGK, kb = idx % kGK;
      const int j = j0 + jj, k = k0 + kb;
      Bs[kb][jj] = (j < N && k < K) ? B[(size_t)j * ldb + k] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kGK; ++kk) {
      const double2 a0 = As[kk][tx], a1 = As[kk][tx + 16];
      const double2 b0 = Bs[kk][ty], b1 = Bs[kk][ty + 16];
      acc[0][0] = cadd(acc[0][0], cmul(a0, b0));
      acc[0][1] = cadd(acc[0][1], cmul(a0, b1));
      acc[1][0] = cadd(acc[1][0], cmul(a1, b0));
      acc[1][1] = cadd(acc[1][1], cmul(a1, b1));
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y) {
      const int i = i0 + tx + 16 * x, j = j0 + ty + 16 * y;
      if (i < M && j < N) C[(size_t)j * ldc + i] = acc[x][y];
    }
}

cudaError_t launch_zgemm_batched(int conj_a, int M, int N, int K, const double2* A, int lda, long long sa,
                                 const double2* B, int ldb, long long sb, double2* C, int ldc, long long sc,
                                 int batch, cudaStream_t st) {
  if (M <= 0 || N <= 0 || batch <= 0) return cudaSuccess;
  if (batch > 65535) return cudaErrorInvalidValue;
  dim3 grid((M + kGT - 1) / kGT, (N + kGT - 1) / kGT, batch);
  zgemm_kernel<<<grid, 256, 0, st>>>(conj_a, M, N, K, A, lda, sa, B, ldb, sb, C, ldc, sc);
  return cudaGetLastError();
}

// ------------------------------------------------------ eigenvector adjoint
__global__ void eig_kmat_kernel(const double2* __restrict__ C, double2* __restrict__ Kout,
                                const double* __restrict__ lam, int lam_stride, const double* __restrict__ lbar,
                                int nall, int ns, int batch, double tau) {
  const long long total = (long long)batch * ns * nall;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(idx % nall);
    const long long bj = idx / nall;
    const int j = (int)(bj % ns);
    const long long b = bj / ns;
    const double* lb = lam + b * lam_stride;
    double2 out = make_double2(0, 0);
    if (m == j) {
      out = make_double2(lbar[b * ns + j], 0.0);
    } else {
      const double gap = lb[j] - lb[m];
      if (fabs(gap) >= tau) {
        const double2 cmj = C[idx];
        if (m < ns) {
          const double2 cjm = C[(b * ns + m) * nall + j];
          out = cscale(csub(cmj, cconj2(cjm)), 0.5 / gap);
        } else {
          out = cscale(cmj, 1.0 / gap);
        }
      }
    }
    Kout[idx] = out;
  }
}

cudaError_t launch_eig_kmat(double2* C, const double* lam, int lam_stride, const double* lbar, int nall, int ns,
                            int batch, double tau, cudaStream_t st) {
  // C holds Z^H Zbar followed (same size) by the output K
  const long long total = (long long)batch * ns * nall;
  if (total <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  eig_kmat_kernel<<<blocks, 256, 0, st>>>(C, C + total, lam, lam_stride, lbar, nall, ns, batch, tau);
  return cudaGetLastError();
}

__global__ void hf_x_kernel(const double2* __restrict__ Z, long long zs, const double* __restrict__ lbar, int n,
                            int ns, int batch, double2* __restrict__ X) {
  const long long total = (long long)batch * ns * n;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % n);
    const long long bj = idx / n;
    const int j = (int)(bj % ns);
    const long long b = bj / ns;
    X[idx] = cscale(Z[b * zs + (long long)j * n + r], lbar[bj]);
  }
}

cudaError_t launch_hf_x(const double2* Z, long long zs, const double* lbar, int n, int ns, int batch, double2* X,
                        cudaStream_t st) {
  const long long total = (long long)batch * ns * n;
  if (total <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  hf_x_kernel<<<blocks, 256, 0, st>>>(Z, zs, lbar, n, ns, batch, X);
  return cudaGetLastError();
}

// ------------------------------------------------------------- resolvent
// Complement part of the eigenvector adjoint without the complement's
// eigenvectors: Y_k += P (lam_k - H)^-1 P zbar_k, P = 1 - Z_S Z_S^H, with
// (lam - H)^-1 = Q (lam - T)^-1 Q^H from the reduction H = Q T Q^H. One warp
// per right-hand side, rows in registers (MAXS slots of 32); the tridiagonal
// solve runs on lane 0. (lam_k - T) is singular along the eigenvectors of S;
// the right-hand side has no component there and the final projection removes
// what rounding puts there.
template <int MAXS>
__global__ void __launch_bounds__(256) resolvent_kernel(ResolventArgs a) {
  const int b = blockIdx.x, n = a.n;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double2* H = a.H + (size_t)b * n * n;
  const double* d = a.tri + (size_t)b * 4 * n;
  const double* e = d + n;
  const double2* tau = reinterpret_cast<const double2*>(d + 2 * n);
  const double2* Z = a.Z + (size_t)b * a.zs;
  __shared__ double s_tiny;
  if (threadIdx.x == 0) {
    double tn = 0.0;
    for (int i = 0; i < n; ++i) {
      const double el = i > 0 ? fabs(e[i - 1]) : 0.0, er = i < n - 1 ? fabs(e[i]) : 0.0;
      tn = fmax(tn, fabs(d[i]) + el + er);
    }
    s_tiny = DBL_EPSILON * fmax(tn, DBL_MIN);
  }
  __syncthreads();
  const double tiny = s_tiny;
  double* u0 = a.work + ((size_t)b * nw + wid) * 5 * n;
  double* u1 = u0 + n;
  double* u2 = u1 + n;
  double* xr = u2 + n;
  double* xi = xr + n;
  auto project = [&](double2* y) {
    for (int m = 0; m < a.nsx; ++m) {
      const double2* zm = Z + (size_t)m * n;
      double2 dot = make_double2(0, 0);
#pragma unroll
      for (int s = 0; s < MAXS; ++s) {
        const int r = 32 * s + lane;
        if (r < n) dot = cadd(dot, cmulc(zm[r], y[s]));
      }
      dot = warp_sum2(dot);
#pragma unroll
      for (int s = 0; s < MAXS; ++s) {
        const int r = 32 * s + lane;
        if (r < n) y[s] = csub(y[s], cmul(zm[r], dot));
      }
    }
  };
  // apply H_j (conj = false) or H_j^H (conj = true): y -= t v (v^H y)
  auto reflect = [&](double2* y, int j, bool conj) {
    double2 t = tau[j];
    if (t.x == 0.0 && t.y == 0.0) return;
    if (conj) t.y = -t.y;
    const double2* v = H + (size_t)j * n;
    double2 dot = make_double2(0, 0);
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      if (32 * s + 31 <= j || 32 * s >= n) continue;  // warp-uniform
      const int r = 32 * s + lane;
      if (r > j && r < n) dot = cadd(dot, cmulc(v[r], y[s]));
    }
    const double2 sc = cmul(t, warp_sum2(dot));
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      if (32 * s + 31 <= j || 32 * s >= n) continue;
      const int r = 32 * s + lane;
      if (r > j && r < n) y[s] = csub(y[s], cmul(v[r], sc));
    }
  };
  for (int k = wid; k < a.ns; k += nw) {
    const double lk = a.lam[(size_t)b * a.lam_stride + k];
    const double2* zb = a.zbar + ((size_t)b * a.ns + k) * n;
    double2 y[MAXS];
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      const int r = 32 * s + lane;
      y[s] = r < n ? zb[r] : make_double2(0, 0);
    }
    project(y);
    for (int j = 0; j < n - 1; ++j) reflect(y, j, true);
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      const int r = 32 * s + lane;
      if (r < n) {
        xr[r] = y[s].x;
        xi[r] = y[s].y;
      }
    }
    __syncwarp();
    if (lane == 0) {
      tri_solve(d, e, n, lk, tiny, xr, u0, u1, u2);
      tri_solve(d, e, n, lk, tiny, xi, u0, u1, u2);
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      const int r = 32 * s + lane;
      y[s] = r < n ? make_double2(-xr[r], -xi[r]) : make_double2(0, 0);
    }
    __syncwarp();
    for (int j = n - 2; j >= 0; --j) reflect(y, j, false);
    project(y);
    double2* out = a.Y + ((size_t)b * a.ns + k) * n;
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      const int r = 32 * s + lane;
      if (r < n) out[r] = cadd(out[r], y[s]);
    }
  }
}

cudaError_t launch_resolvent(const ResolventArgs& a, cudaStream_t st) {
  if (a.nitems <= 0 || a.ns <= 0) return cudaSuccess;
  const int slots = (a.n + 31) / 32;
#define PMX_RES(S)                                                  \
  if (slots <= S) {                                                 \
    resolvent_kernel<S><<<a.nitems, 256, 0, st>>>(a);               \
    return cudaGetLastError();                                      \
  }
  PMX_RES(4)
  PMX_RES(9)
  PMX_RES(13)
  PMX_RES(19)
  PMX_RES(26)
  PMX_RES(38)
#undef PMX_RES
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------- pair accumulators
namespace {
constexpr int kHT = 16, kHJ = 8;
}

template <bool SOC>
__global__ void __launch_bounds__(256) hgrad_kernel(const double2* __restrict__ X, long long xs,
                                                    const double2* __restrict__ Z, long long zs,
                                                    const double* __restrict__ kpts, int batch, int n, int npw,
                                                    int ns, double2* __restrict__ R) {
  constexpr int W = SOC ? 2 : 1;  // components per plane wave
  __shared__ double2 Xs[kHJ][kHT * W];
  __shared__ double2 Zs[kHJ][kHT * W];
  const int tid = threadIdx.x, ti = tid % kHT, tj = tid / kHT;
  const int i0 = blockIdx.x * kHT, j0 = blockIdx.y * kHT;
  constexpr int NS = SOC ? 4 : 1, NW = SOC ? 4 : 1;
  double2 acc[NW][NS];
#pragma unroll
  for (int w = 0; w < NW; ++w)
#pragma unroll
    for (int s = 0; s < NS; ++s) acc[w][s] = make_double2(0, 0);
  for (int b = 0; b < batch; ++b) {
    double2 P[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) P[s] = make_double2(0, 0);
    const double2* Xb = X + (size_t)b * xs;
    const double2* Zb = Z + (size_t)b * zs;
    for (int s0 = 0; s0 < ns; s0 += kHJ) {
      for (int idx = tid; idx < 2 * kHJ * kHT * W; idx += 256) {
        const int which = idx / (kHJ * kHT * W);
        const int rem = idx % (kHJ * kHT * W);
        const int jj = rem / (kHT * W), cc = rem % (kHT * W);
        const int st = s0 + jj;
        if (which == 0) {
          const int r = i0 * W + cc;
          Xs[jj][cc] = (st < ns && r < n) ? Xb[(size_t)st * n + r] : make_double2(0, 0);
        } else {
          const int r = j0 * W + cc;
          Zs[jj][cc] = (st < ns && r < n) ? Zb[(size_t)st * n + r] : make_double2(0, 0);
        }
      }
      __syncthreads();
#pragma unroll
      for (int jj = 0; jj < kHJ; ++jj) {
        if (SOC) {
          const double2 x0 = Xs[jj][2 * ti], x1 = Xs[jj][2 * ti + 1];
          const double2 z0 = Zs[jj][2 * tj], z1 = Zs[jj][2 * tj + 1];
          P[0] = cadd(P[0], cmulc(x0, z0));
          P[NS > 1 ? 1 : 0] = cadd(P[NS > 1 ? 1 : 0], cmulc(x0, z1));
          P[NS > 2 ? 2 : 0] = cadd(P[NS > 2 ? 2 : 0], cmulc(x1, z0));
          P[NS > 3 ? 3 : 0] = cadd(P[NS > 3 ? 3 : 0], cmulc(x1, z1));
        } else {
          P[0] = cadd(P[0], cmulc(Xs[jj][ti], Zs[jj][tj]));
        }
      }
      __syncthreads();
    }
    if (SOC) {
      const double wt[4] = {1.0, kpts[3 * b], kpts[3 * b + 1], kpts[3 * b + 2]};
#pragma unroll
      for (int w = 0; w < NW; ++w)
#pragma unroll
        for (int s = 0; s < NS; ++s) acc[w][s] = cadd(acc[w][s], cscale(P[s], wt[w]));
    } else {
      acc[0][0] = cadd(acc[0][0], P[0]);
    }
  }
  const int i = i0 + ti, j = j0 + tj;
  if (i < npw && j < npw) {
    const size_t pl = (size_t)npw * npw;
#pragma unroll
    for (int w = 0; w < NW; ++w)
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        double2* r = R + (size_t)(w * NS + s) * pl + (size_t)i * npw + j;
        *r = cadd(*r, acc[w][s]);
      }
  }
}

cudaError_t launch_hgrad(const double2* X, long long xs, const double2* Z, long long zs, const double* kpts,
                         int batch, int n, int npw, int soc, int ns, double2* R, cudaStream_t st) {
  if (batch <= 0 || npw <= 0) return cudaSuccess;
  dim3 grid((npw + kHT - 1) / kHT, (npw + kHT - 1) / kHT);
  if (soc)
    hgrad_kernel<true><<<grid, 256, 0, st>>>(X, xs, Z, zs, kpts, batch, n, npw, ns, R);
  else
    hgrad_kernel<false><<<grid, 256, 0, st>>>(X, xs, Z, zs, kpts, batch, n, npw, ns, R);
  return cudaGetLastError();
}

__global__ void hscatter_kernel(const double2* __restrict__ R, int npw, int soc, const int* __restrict__ hkl,
                                const double* __restrict__ G, int imax, double2* __restrict__ SV,
                                double2* __restrict__ SSO) {
  const long long total = (long long)npw * npw;
  const int off = 2 * imax, side = 4 * imax + 1;
  const size_t pl = (size_t)npw * npw;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / npw), j = (int)(idx % npw);
    if (i == j) continue;
    const int dh = hkl[3 * i] - hkl[3 * j], dk = hkl[3 * i + 1] - hkl[3 * j + 1], dl = hkl[3 * i + 2] - hkl[3 * j + 2];
    const size_t d = ((size_t)(dh + off) * side + (dk + off)) * side + (dl + off);
    const size_t dp = ((size_t)(-dh + off) * side + (-dk + off)) * side + (-dl + off);
    if (!soc) {
      const double2 v = R[idx];
      atomicAdd(&SV[d].x, v.x);
      atomicAdd(&SV[d].y, v.y);
      continue;
    }
    auto Rw = [&](int w, int s) { return R[(size_t)(w * 4 + s) * pl + idx]; };
    const double2 v = cadd(Rw(0, 0), Rw(0, 3));
    atomicAdd(&SV[d].x, v.x);
    atomicAdd(&SV[d].y, v.y);
    // Pauli components T^x_w = sum_ss' R[w][ss'] sigma^x_ss'
    double2 T[3][4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const double2 r0 = Rw(w, 0), r1 = Rw(w, 1), r2 = Rw(w, 2), r3 = Rw(w, 3);
      T[0][w] = cadd(r1, r2);
      // -i r1 + i r2
      T[1][w] = make_double2(r1.y - r2.y, -r1.x + r2.x);
      T[2][w] = csub(r0, r3);
    }
    const double* Gi = G + 3 * i;
    const double* Gj = G + 3 * j;
    // a = G_j x G_i ; dG = G_i - G_j
    const double ax = Gj[1] * Gi[2] - Gj[2] * Gi[1];
    const double ay = Gj[2] * Gi[0] - Gj[0] * Gi[2];
    const double az = Gj[0] * Gi[1] - Gj[1] * Gi[0];
    const double g0 = Gi[0] - Gj[0], g1 = Gi[1] - Gj[1], g2 = Gi[2] - Gj[2];
    double2 S = cadd(cadd(cscale(T[0][0], ax), cscale(T[1][0], ay)), cscale(T[2][0], az));
    // sum_xyz eps_xyz dG_z T^x_{y+1}
    S = cadd(S, csub(cscale(T[0][2], g2), cscale(T[0][3], g1)));
    S = cadd(S, csub(cscale(T[1][3], g0), cscale(T[1][1], g2)));
    S = cadd(S, csub(cscale(T[2][1], g1), cscale(T[2][2], g0)));
    // SSO += i S
    atomicAdd(&SSO[dp].x, -S.y);
    atomicAdd(&SSO[dp].y, S.x);
  }
}

cudaError_t launch_hscatter(const double2* R, int npw, int soc, const int* hkl, const double* G, int imax,
                            double2* SV, double2* SSO, cudaStream_t st) {
  const long long total = (long long)npw * npw;
  if (total <= 0) return cudaSuccess;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  hscatter_kernel<<<blocks, 256, 0, st>>>(R, npw, soc, hkl, G, imax, SV, SSO);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmx
