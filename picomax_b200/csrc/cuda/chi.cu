// Stage 2 kernels, FP64 path: overlaps, delta-weighted contraction, scaling and
// the Kramers-Kronig transform of chi_tensor (src/pmx_chi.cpp:319-713) and
// chi_LL (src/pmx_chi_copy.cpp:320-676).
//
// Layouts
//   eigenvectors: z[item][s][row], rows interleaved (G0 up, G0 down, ...) with SOC,
//                 plain G order without SOC (spatial states, spectrum doubled).
//   M[t][a][ch]:  overlap of transition t (sorted), a = 3 m + i (i: L, T+, T-),
//                 ch = channel (1 for epsLL and spin-free epsij, 4 for epsij with
//                 SOC: up, down, updown, downup as in src/pmx_chi.cpp:534-544).
//   acc[2][9][np][nf]: Re then Im accumulators per (i, j, pair(m, n<=m), f),
//                 pair(m, n) = m(m+1)/2 + n, which is the .dat order for one q.
#include <cfloat>
#include <cmath>

#include "pmx_chi.hpp"
#include "pmx_common.cuh"

namespace pmx {
namespace dev {

// ------------------------------------------------------------------- overlaps
// One CTA per (k, conduction chunk, valence chunk), the chunks' eigenvectors
// staged in shared memory (rows padded by 16 bytes). Each thread owns one
// (m, c, v) task at a time (pairs fastest, so a warp shares m and its loci
// row) and sums over the plane waves p with loci[m][p] != -1, accumulating
// the moments sum_p conj(c(p)) v(loci p) {1, G_p.x, G_p.y, G_p.z} per spin
// channel in registers: no cross-lane reductions. The
// orbital current u_i^H (G_p + k + q/2 + G_m/2) and the SOC current
// u_i^H v_soc(G_m) (src/pmx_chi.cpp:203-266, constant over p because
// G_loci - G_p = G_m) are then applied to the moments.
__global__ void __launch_bounds__(256) overlap_kernel(OverlapArgs a) {
  const int k = blockIdx.x;
  const int ncd = a.ncd[k], nvd = a.nvd[k];
  // blockIdx.y = (conduction chunk) + ncc * (valence chunk)
  const int ncc = (a.ncd_max + a.cchunk - 1) / a.cchunk;
  const int c_lo = (blockIdx.y % ncc) * a.cchunk;
  const int c_hi = min(ncd, c_lo + a.cchunk);
  const int v_lo = (blockIdx.y / ncc) * a.vchunk;
  const int v_hi = min(nvd, v_lo + a.vchunk);
  if (c_lo >= c_hi || v_lo >= v_hi) return;
  const int nvl = v_hi - v_lo;
  const int n = a.n, npw = a.npw, ldn = n + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* sc = reinterpret_cast<double2*>(smraw);           // [cchunk][ldn]
  double2* sv = sc + (size_t)a.cchunk * ldn;                  // [vchunk][ldn]
  double* sg = reinterpret_cast<double*>(sv + (size_t)a.vchunk * ldn);  // [npw][3]
  const int tid = threadIdx.x;
  for (int c = c_lo; c < c_hi; ++c) {
    const double2* src = a.zk + ((size_t)k * a.nev + a.cidx[a.cbase[k] + c]) * n;
    for (int r = tid; r < n; r += blockDim.x) sc[(size_t)(c - c_lo) * ldn + r] = src[r];
  }
  for (int v = v_lo; v < v_hi; ++v) {
    const double2* src = a.zq + ((size_t)k * a.nev + a.vidx[a.vbase[k] + v]) * n;
    for (int r = tid; r < n; r += blockDim.x) sv[(size_t)(v - v_lo) * ldn + r] = src[r];
  }
  for (int r = tid; r < 3 * npw; r += blockDim.x) sg[r] = a.G[r];
  __syncthreads();
  const double kx = a.kpts[3 * k], ky = a.kpts[3 * k + 1], kz = a.kpts[3 * k + 2];
  const int npair = (c_hi - c_lo) * nvl;
  const int A = 3 * a.neps;
  const int ntask = a.neps * npair;
  for (int task = tid; task < ntask; task += blockDim.x) {
    const int m = task / npair, pr = task - m * npair;
    const int cl = pr / nvl, v = v_lo + pr % nvl;
    const long long dst = a.dest[a.blkoff[k] + (long long)(c_lo + cl) * nvd + v];
    if (dst < 0) continue;
    const int* loci = a.loci + (size_t)m * npw;
    const double2* cvec = sc + (size_t)cl * ldn;
    const double2* vvec = sv + (size_t)(v - v_lo) * ldn;
    // moments: [0..3] spin-summed or up-up, [4..7] down-down, [8] up-down, [9] down-up
    double2 mo[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) mo[q] = make_double2(0, 0);
    for (int p = 0; p < npw; ++p) {
      const int lp = loci[p];
      if (lp < 0) continue;
      const double gx = sg[3 * p], gy = sg[3 * p + 1], gz = sg[3 * p + 2];
      if (!a.soc) {
        const double2 s = cmulc(cvec[p], vvec[lp]);
        mo[0] = cadd(mo[0], s);
        mo[1] = cadd(mo[1], cscale(s, gx));
        mo[2] = cadd(mo[2], cscale(s, gy));
        mo[3] = cadd(mo[3], cscale(s, gz));
      } else {
        const double2 cu = cvec[2 * p], cd = cvec[2 * p + 1];
        const double2 vu = vvec[2 * lp], vd = vvec[2 * lp + 1];
        const double2 uu = cmulc(cu, vu), dd = cmulc(cd, vd);
        if (a.nch == 4) {
          mo[0] = cadd(mo[0], uu);
          mo[1] = cadd(mo[1], cscale(uu, gx));
          mo[2] = cadd(mo[2], cscale(uu, gy));
          mo[3] = cadd(mo[3], cscale(uu, gz));
          mo[4] = cadd(mo[4], dd);
          mo[5] = cadd(mo[5], cscale(dd, gx));
          mo[6] = cadd(mo[6], cscale(dd, gy));
          mo[7] = cadd(mo[7], cscale(dd, gz));
          mo[8] = cadd(mo[8], cmulc(cu, vd));
          mo[9] = cadd(mo[9], cmulc(cd, vu));
        } else {
          const double2 s = cadd(uu, dd);
          mo[0] = cadd(mo[0], s);
          mo[1] = cadd(mo[1], cscale(s, gx));
          mo[2] = cadd(mo[2], cscale(s, gy));
          mo[3] = cadd(mo[3], cscale(s, gz));
        }
      }
    }
    // w = k + q/2 + G_m/2, as in (G_p + K + Q/2 + G_m/2) at src/pmx_chi.cpp:535
    const double wx = (kx + a.q[0] / 2) + a.G[3 * m] / 2;
    const double wy = (ky + a.q[1] / 2) + a.G[3 * m + 1] / 2;
    const double wz = (kz + a.q[2] / 2) + a.G[3 * m + 2] / 2;
    double2* out = a.M + ((size_t)dst * A + 3 * m) * a.nch;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
      const double2* u = a.uvec + ((size_t)m * 3 + i) * 3;  // u_i of q+G_m
      const double2 s = a.ssoc[m * 3 + i];                  // u_i^H v_soc(G_m)
      // orbital current of a moment set: sum_x conj(u_x) (M_x + w_x M_0)
      auto orb = [&](const double2* mm) {
        double2 r = cmulc(u[0], cadd(mm[1], cscale(mm[0], wx)));
        r = cadd(r, cmulc(u[1], cadd(mm[2], cscale(mm[0], wy))));
        r = cadd(r, cmulc(u[2], cadd(mm[3], cscale(mm[0], wz))));
        return r;
      };
      if (a.mode == 1) {  // epsLL: L = density, T = u.(v_orb + v_soc)
        out[(size_t)i * a.nch] = i == 0 ? mo[0] : cadd(orb(mo), cmul(s, mo[0]));
      } else if (a.nch == 1) {  // epsij without SOC: single channel, orbital current
        out[(size_t)i * a.nch] = orb(mo);
      } else {  // epsij with SOC: up, down, updown, downup
        double2* o = out + (size_t)i * 4;
        o[0] = orb(mo);
        o[1] = orb(mo + 4);
        o[2] = cmul(s, mo[8]);
        o[3] = cmul(s, mo[9]);
      }
    }
  }
}

cudaError_t launch_overlap(const OverlapArgs& a, int nk, cudaStream_t st) {
  if (nk <= 0) return cudaSuccess;
  if (a.cchunk < 1 || a.vchunk < 1) return cudaErrorInvalidValue;
  const size_t smem = overlap_smem_bytes(a.cchunk, a.vchunk, a.n, a.npw);
  cudaError_t err = cudaFuncSetAttribute(overlap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  const int ncc = (a.ncd_max + a.cchunk - 1) / a.cchunk, nvc = (a.nvd_max + a.vchunk - 1) / a.vchunk;
  dim3 grid(nk, ncc * nvc);
  overlap_kernel<<<grid, 256, smem, st>>>(a);
  return cudaGetLastError();
}

size_t overlap_smem_bytes(int cchunk, int vchunk, int n, int npw) {
  return ((size_t)cchunk + vchunk) * (n + 1) * sizeof(double2) + (size_t)3 * npw * sizeof(double);
}

bool overlap_tiles(int ncd_max, int nvd_max, int n, int npw, int& cchunk, int& vchunk) {
  const size_t lim = 200 * 1024;
  vchunk = std::max(1, nvd_max);
  cchunk = std::max(1, ncd_max);
  while (cchunk > 1 && overlap_smem_bytes(cchunk, vchunk, n, npw) > lim) --cchunk;
  while (vchunk > 1 && overlap_smem_bytes(cchunk, vchunk, n, npw) > lim) --vchunk;
  return overlap_smem_bytes(cchunk, vchunk, n, npw) <= lim;
}

int overlap_tile_candidates(int ncd_max, int nvd_max, int n, int npw, int* cc, int* vc, int maxc) {
  int c0 = 1, v0 = 1;
  if (!overlap_tiles(ncd_max, nvd_max, n, npw, c0, v0) || maxc < 1) return 0;
  const int cs[2] = {c0, (c0 + 1) / 2}, vs[2] = {v0, (v0 + 1) / 2};
  int cnt = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      bool dup = false;
      for (int q = 0; q < cnt; ++q) dup = dup || (cc[q] == cs[i] && vc[q] == vs[j]);
      if (!dup && cnt < maxc) {
        cc[cnt] = cs[i];
        vc[cnt] = vs[j];
        ++cnt;
      }
    }
  return cnt;
}

// ------------------------------------------------------------ broadening
// src/pmx_chi.cpp:90-164; delta model 0 gauss, 1 lorentz, 2 triangle, 3 rect.
__device__ __forceinline__ double broaden(int model, double eps, double x) {
  switch (model) {
    case 0:
      return exp(-0.5 * x * x / (eps * eps)) / (eps * sqrt(2.0 * 3.14159265358979323846));
    case 1:
      return eps / 3.14159265358979323846 / (eps * eps + x * x);
    case 2:
      return fabs(x) < 0.5 * eps ? 4.0 / eps * (0.5 - fabs(x) / eps) : 0.0;
    default:
      return fabs(x) < 0.5 * eps ? 1.0 / eps : 0.0;
  }
}

// ------------------------------------------------------- FP64 contraction
// acc_im[p,f] = sum_t w_t reO_t(p) delta(dE_t - w_f), acc_re[p,f] = -sum_t w_t imO_t(p) delta(...)
// over the transitions whose window covers f (src/pmx_chi.cpp:573-627) or over
// all transitions (src/pmx_chi_copy.cpp:546-575). One CTA computes a 12x12
// block of (a, b) = (3m+i, 3n+j) pairs for 64 frequencies; the tile's
// transition range is contiguous because transitions are sorted by window start.
namespace {
constexpr int kMB = 4;              // m per block
constexpr int kAB = 3 * kMB;        // a (or b) per block
constexpr int kPairs = kAB * kAB;   // 144
constexpr int kFT = 64;             // frequencies per tile
constexpr int kTK = 16;             // transitions per chunk
constexpr int kCThreads = 256;
}  // namespace

__device__ __forceinline__ void tile_of(int id, int& ta, int& tb) {
  // lower-triangular enumeration: id -> (ta >= tb)
  int r = (int)((sqrt(8.0 * id + 1.0) - 1.0) * 0.5);
  while ((r + 1) * (r + 2) / 2 <= id) ++r;
  while (r * (r + 1) / 2 > id) --r;
  ta = r;
  tb = id - r * (r + 1) / 2;
}

template <int NCH, bool PV>
__global__ void __launch_bounds__(kCThreads) contract_f64_kernel(ContractArgs a) {
  int ta, tb;
  tile_of(blockIdx.x, ta, tb);
  const int f_lo = blockIdx.y * kFT;
  const int2 tr = a.trange[blockIdx.y];
  const int A = 3 * a.neps;
  const int a0 = ta * kAB, b0 = tb * kAB;
  extern __shared__ __align__(16) unsigned char smraw[];
  typedef double2 MTile[kAB][NCH];
  typedef double PRow[kTK + 1];
  typedef double WTile[kTK][kFT];
  MTile* sMa = reinterpret_cast<MTile*>(smraw);
  MTile* sMb = sMa + kTK;
  PRow* sP1 = reinterpret_cast<PRow*>(sMb + kTK);
  PRow* sP2 = sP1 + kPairs;
  WTile* sW = reinterpret_cast<WTile*>(sP2 + kPairs);
  double* sw = reinterpret_cast<double*>(sW + (PV ? 4 : 1));
  double* sde = sw + kTK;
  int* sf0 = reinterpret_cast<int*>(sde + kTK);
  const int tid = threadIdx.x;
  const int pg = tid / 16, fg = tid % 16;
  double acc1[9][4], acc2[9][4];  // 1: Im (reO), 2: Re (-imO)
  double pv1[PV ? 9 : 1][4], pv2[PV ? 9 : 1][4];
#pragma unroll
  for (int u = 0; u < 9; ++u)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      acc1[u][q] = 0;
      acc2[u][q] = 0;
      if (PV) {
        pv1[u][q] = 0;
        pv2[u][q] = 0;
      }
    }
  int pclass[9];
#pragma unroll
  for (int u = 0; u < 9; ++u) {
    const int pp = pg * 9 + u;
    const int i = (pp / kAB) % 3, j = (pp % kAB) % 3;
    pclass[u] = a.pvclass ? a.pvclass : ((i == 0 && j == 0) ? 1 : ((i == 0 || j == 0) ? 2 : 3));
  }
  for (int t0 = tr.x; t0 < tr.y; t0 += kTK) {
    const int nt = min(kTK, tr.y - t0);
    // stage M of the chunk
    for (int idx = tid; idx < kTK * kAB * NCH; idx += kCThreads) {
      const int t = idx / (kAB * NCH), rem = idx % (kAB * NCH);
      const int aa = rem / NCH, ch = rem % NCH;
      double2 va = make_double2(0, 0), vb = make_double2(0, 0);
      if (t < nt) {
        const size_t base = (size_t)(t0 + t) * A * NCH;
        if (a0 + aa < A) va = a.M[base + (size_t)(a0 + aa) * NCH + ch];
        if (b0 + aa < A) vb = a.M[base + (size_t)(b0 + aa) * NCH + ch];
      }
      sMa[t][aa][ch] = va;
      sMb[t][aa][ch] = vb;
    }
    if (tid < kTK) {
      const int t = tid;
      sw[t] = t < nt ? a.wgt[t0 + t] : 0.0;
      sde[t] = t < nt ? a.dE[t0 + t] : 0.0;
      sf0[t] = t < nt ? a.f0[t0 + t] : 0;
    }
    __syncthreads();
    // pair products P1 = w reO, P2 = -w imO
    for (int idx = tid; idx < kPairs * kTK; idx += kCThreads) {
      const int pp = idx / kTK, t = idx % kTK;
      const int ia = pp / kAB, ib = pp % kAB;
      double reO, imO;
      if (NCH == 1) {
        const double2 o = cmulc(sMb[t][ib][0], sMa[t][ia][0]);  // a conj(b)
        reO = o.x;
        imO = o.y;
      } else {
        const double2 up_a = sMa[t][ia][0], dn_a = sMa[t][ia][1], ud_a = sMa[t][ia][2], du_a = sMa[t][ia][3];
        const double2 up_b = sMb[t][ib][0], dn_b = sMb[t][ib][1], ud_b = sMb[t][ib][2], du_b = sMb[t][ib][3];
        double2 tt = cmulc(up_b, up_a);
        tt = cadd(tt, cmulc(dn_b, dn_a));
        tt = csub(tt, cmulc(ud_b, ud_a));
        tt = csub(tt, cmulc(du_b, du_a));
        double2 cr = cmulc(dn_b, up_a);
        cr = cadd(cr, cmulc(up_b, dn_a));
        cr = csub(cr, cmulc(ud_b, du_a));
        cr = csub(cr, cmulc(du_b, ud_a));
        reO = tt.x + cr.x;
        imO = tt.y;
      }
      sP1[pp][t] = sw[t] * reO;
      sP2[pp][t] = -sw[t] * imO;
    }
    // weights
    for (int idx = tid; idx < kTK * kFT; idx += kCThreads) {
      const int t = idx / kFT, fl = idx % kFT;
      const int f = f_lo + fl;
      double wv = 0.0;
      const bool in = t < nt && f < a.nf && (a.window < 0 || abs(f - sf0[t]) <= a.window);
      const double om = a.dfreq * f;
      if (in) wv = broaden(a.delta, a.eps, sde[t] - om);
      sW[0][t][fl] = wv;
      if (PV) {
        const double de = sde[t];
        const double den = de * de - om * om;
        const bool ok = t < nt && f < a.nf;
        sW[1][t][fl] = ok ? de / den : 0.0;          // LL
        sW[2][t][fl] = ok ? 1.0 / den : 0.0;         // LT
        sW[3][t][fl] = ok ? 1.0 / de / den : 0.0;    // TT
      }
    }
    __syncthreads();
    for (int t = 0; t < nt; ++t) {
      double wv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) wv[q] = sW[0][t][fg + 16 * q];
#pragma unroll
      for (int u = 0; u < 9; ++u) {
        const double p1 = sP1[pg * 9 + u][t], p2 = sP2[pg * 9 + u][t];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc1[u][q] = fma(p1, wv[q], acc1[u][q]);
          acc2[u][q] = fma(p2, wv[q], acc2[u][q]);
        }
        if (PV) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double g = sW[pclass[u]][t][fg + 16 * q];
            pv1[u][q] = fma(p1, g, pv1[u][q]);   // Re2 += w Re(O) g
            pv2[u][q] = fma(-p2, g, pv2[u][q]);  // Im2 += w Im(O) g
          }
        }
      }
    }
    __syncthreads();
  }
  // store
  const size_t blk = (size_t)9 * a.np * a.nf;
#pragma unroll
  for (int u = 0; u < 9; ++u) {
    const int pp = pg * 9 + u;
    const int ia = pp / kAB, ib = pp % kAB;
    const int av = a0 + ia, bv = b0 + ib;
    const int m = av / 3, i = av % 3, nn = bv / 3, j = bv % 3;
    if (m >= a.neps || nn >= a.neps || nn > m) continue;
    const size_t row = ((size_t)(i * 3 + j) * a.np + (size_t)m * (m + 1) / 2 + nn) * a.nf;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int f = f_lo + fg + 16 * q;
      if (f >= a.nf) continue;
      a.acc[row + f] = acc2[u][q];        // Re part
      a.acc[blk + row + f] = acc1[u][q];  // Im part
      if (PV) {
        a.acc_pv[row + f] = pv1[u][q];
        a.acc_pv[blk + row + f] = pv2[u][q];
      }
    }
  }
}

cudaError_t launch_contract_f64(const ContractArgs& a, cudaStream_t st) {
  const int nmb = (a.neps + kMB - 1) / kMB;
  const int ntiles = nmb * (nmb + 1) / 2;
  const int nft = (a.nf + kFT - 1) / kFT;
  dim3 grid(ntiles, nft);
  const bool pv = a.acc_pv != nullptr;
  auto smem = [](int nch, bool p) {
    return (size_t)2 * kTK * kAB * nch * sizeof(double2) + (size_t)2 * kPairs * (kTK + 1) * sizeof(double) +
           (size_t)(p ? 4 : 1) * kTK * kFT * sizeof(double) + (size_t)2 * kTK * sizeof(double) +
           (size_t)kTK * sizeof(int);
  };
  cudaError_t err;
#define PMX_LAUNCH_CONTRACT(NCH_, PV_)                                                              \
  {                                                                                                 \
    const size_t sm = smem(NCH_, PV_);                                                              \
    err = cudaFuncSetAttribute(contract_f64_kernel<NCH_, PV_>,                                       \
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);               \
    if (err != cudaSuccess) return err;                                                             \
    contract_f64_kernel<NCH_, PV_><<<grid, kCThreads, sm, st>>>(a);                                 \
  }
  if (a.nch == 1) {
    if (pv)
      PMX_LAUNCH_CONTRACT(1, true)
    else
      PMX_LAUNCH_CONTRACT(1, false)
  } else {
    if (pv) return cudaErrorInvalidValue;
    PMX_LAUNCH_CONTRACT(4, false)
  }
#undef PMX_LAUNCH_CONTRACT
  return cudaGetLastError();
}

int contract_ftile() { return kFT; }

// ---------------------------------------------------------------- scaling
// epsij: chi = SCALEFACTOR acc / w_f^2 with 1/w_0^2 := 0 (src/pmx_chi.cpp:559-563, :631-634).
// epsLL: chi = pi acc * class factor (src/pmx_chi_copy.cpp:579-596), f = 0 gives 0,
//        plus 2 * PV * class factor when kk = 0 (:597-615).
__global__ void scale_kernel(ScaleArgs s) {
  const size_t blk = (size_t)9 * s.np * s.nf;
  const size_t total = 2 * blk;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const size_t r = idx % blk;
    const int f = (int)(r % s.nf);
    const size_t row = r / s.nf;
    const int pair = (int)(row % s.np);
    const int ij = (int)(row / s.np);
    const int i = ij / 3, j = ij % 3;
    int m = (int)((sqrt(8.0 * pair + 1.0) - 1.0) * 0.5);
    while ((m + 1) * (m + 2) / 2 <= pair) ++m;
    while (m * (m + 1) / 2 > pair) --m;
    const int n = pair - m * (m + 1) / 2;
    const double w = s.dfreq * f;
    double v = s.acc[idx];
    if (s.mode == 0) {
      const double inv = f == 0 ? 0.0 : 1.0 / (w * w);
      v = s.sf * (v * inv);
    } else {
      const double qm = s.qgn[m], qn = s.qgn[n];
      double f1;
      if (f == 0) {
        f1 = 0.0;
      } else if (s.mode == 2) {  // epsxyz: every block scales as TT (src/pmx_chi_copy.cpp:1093, :1272-1281)
        f1 = s.sf_tt / (w * w);
      } else if (i == 0 && j == 0) {
        f1 = s.sf_ll / (qm * qn);
      } else if (i == 0) {
        f1 = s.sf_lt / (qm * w);
      } else if (j == 0) {
        f1 = s.sf_lt / qn;
      } else {
        f1 = s.sf_tt / (w * w);
      }
      double out = 3.14159265358979323846 * (v * f1);
      if (s.acc_pv) {
        double f2;
        if (s.mode == 2)
          f2 = s.sf_tt;
        else if (i == 0 && j == 0)
          f2 = s.sf_ll / (qm * qn);
        else if (i == 0)
          f2 = s.sf_lt / qm;
        else if (j == 0)
          f2 = s.sf_lt / qn;
        else
          f2 = s.sf_tt;
        out += 2.0 * (s.acc_pv[idx] * f2);
      }
      v = out;
    }
    s.out[idx] = v;
  }
}

cudaError_t launch_scale(const ScaleArgs& s, cudaStream_t st) {
  scale_kernel<<<1184, 256, 0, st>>>(s);
  return cudaGetLastError();
}

// ------------------------------------------------------- Kramers-Kronig
// src/pmx_chi.cpp:272-309: Re_f += ds sum_{s!=f} w_s Im_s/(w_s^2-w_f^2),
// Im_f += ds sum_{s!=f} w_s Re0_s/(w_s^2-w_f^2), ds = 2 dw / pi, both from the
// values before the transform. As a GEMM: Y = X K^T with X = [Im; Re] rows and
// K generated on the fly, then chi += ds Y (swapped halves).
namespace {
constexpr int kKT = 64, kKK = 16;
}

__global__ void __launch_bounds__(256) kk_kernel(const double* __restrict__ chi, double* __restrict__ out,
                                                 int rows, int nf, double dfreq) {
  // chi: [2][rows][nf] (Re block then Im block); out same layout.
  const int r0 = blockIdx.x * kKT, f0 = blockIdx.y * kKT;
  __shared__ double sX[kKK][kKT + 1];
  __shared__ double sK[kKK][kKT + 1];
  const int tid = threadIdx.x, tr = tid / 16, tc = tid % 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0;
  const size_t blk = (size_t)rows * nf;
  // logical row r in [0, 2 rows): r < rows -> source Im row r (updates Re), else source Re row
  for (int s0 = 0; s0 < nf; s0 += kKK) {
    for (int idx = tid; idx < kKK * kKT; idx += 256) {
      const int ss = idx / kKT, rr = idx % kKT;
      const int r = r0 + rr, s = s0 + ss;
      double x = 0.0;
      if (r < 2 * rows && s < nf) {
        const size_t src = r < rows ? blk + (size_t)r * nf + s : (size_t)(r - rows) * nf + s;
        x = chi[src];
      }
      sX[ss][rr] = x;
      const int f = f0 + rr;
      double kv = 0.0;
      if (s < nf && f < nf && s != f) {
        const double ws = dfreq * s, wf = dfreq * f;
        kv = ws / (ws * ws - wf * wf);
      }
      sK[ss][rr] = kv;
    }
    __syncthreads();
#pragma unroll
    for (int ss = 0; ss < kKK; ++ss) {
      double xa[4], kb[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) xa[a] = sX[ss][tr + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) kb[b] = sK[ss][tc + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(xa[a], kb[b], acc[a][b]);
    }
    __syncthreads();
  }
  const double ds = dfreq * 2.0 / 3.14159265358979323846;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int r = r0 + tr + 16 * a;
    if (r >= 2 * rows) continue;
    const size_t dst = r < rows ? (size_t)r * nf : blk + (size_t)(r - rows) * nf;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int f = f0 + tc + 16 * b;
      if (f >= nf) continue;
      out[dst + f] = chi[dst + f] + ds * acc[a][b];
    }
  }
}

cudaError_t launch_kk(const double* chi, double* out, int rows, int nf, double dfreq, cudaStream_t st) {
  dim3 grid((2 * rows + kKT - 1) / kKT, (nf + kKT - 1) / kKT);
  kk_kernel<<<grid, 256, 0, st>>>(chi, out, rows, nf, dfreq);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmx

namespace pmx {
namespace dev {

// ------------------------------------------------------------ macroscopic eps
// eps_M(q, w) = 1 / [eps^-1]_00 with eps_mn = delta_mn + chi^LL_mn and the
// n > m half filled by conj(eps_nm), as in the reference's post-processing
// (include/matlab_wrapper/+picomax/+eps/macroscopic.m:13-29, :79). One warp
// per (q, w): Gaussian elimination with partial pivoting of eps x = e_0 in
// shared memory; [eps^-1]_00 = x_0.
__global__ void __launch_bounds__(128) epsm_kernel(const double* __restrict__ re, const double* __restrict__ im,
                                                   int neps, int nq, int nf, double2* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int job = blockIdx.x * (blockDim.x >> 5) + w;
  if (job >= nq * nf) return;
  const int q = job / nf, f = job % nf;
  const int n = neps, ld = n + 1;
  double2* E = reinterpret_cast<double2*>(smraw) + (size_t)w * n * ld;  // row-major, column n = rhs
  const int np = n * (n + 1) / 2;
  // chi LL block: [i=0][j=0][q][pair][f]
  for (int idx = lane; idx < n * n; idx += 32) {
    const int r = idx / n, c = idx % n;
    const int m = r > c ? r : c, nn = r > c ? c : r;
    const size_t o = ((size_t)q * np + (size_t)m * (m + 1) / 2 + nn) * nf + f;
    double2 v = make_double2(re[o], im[o]);
    if (r < c) v.y = -v.y;  // eps_nm = conj(eps_mn) above the diagonal
    if (r == c) v.x += 1.0;
    E[r * ld + c] = v;
  }
  for (int r = lane; r < n; r += 32) E[r * ld + n] = make_double2(r == 0 ? 1.0 : 0.0, 0.0);
  __syncwarp();
  for (int k = 0; k < n; ++k) {
    // pivot search (lane-strided, then warp argmax)
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
      for (int c = lane; c <= n; c += 32) {
        const double2 t = E[k * ld + c];
        E[k * ld + c] = E[bi * ld + c];
        E[bi * ld + c] = t;
      }
    __syncwarp();
    const double2 p = E[k * ld + k];
    const double pd = p.x * p.x + p.y * p.y;
    const double2 inv = make_double2(p.x / pd, -p.y / pd);
    for (int r = k + 1; r < n; ++r) {
      const double2 fct = cmul(E[r * ld + k], inv);
      for (int c = k + lane; c <= n; c += 32) E[r * ld + c] = csub(E[r * ld + c], cmul(fct, E[k * ld + c]));
    }
    __syncwarp();
  }
  if (lane == 0) {
    // back substitution for x_0 only needs the full solve; do it serially
    double2 x[64];
    for (int r = n - 1; r >= 0; --r) {
      double2 s = E[r * ld + n];
      for (int c = r + 1; c < n; ++c) s = csub(s, cmul(E[r * ld + c], x[c]));
      const double2 d = E[r * ld + r];
      const double dd = d.x * d.x + d.y * d.y;
      x[r] = cmul(s, make_double2(d.x / dd, -d.y / dd));
    }
    const double2 x0 = x[0];
    const double xx = x0.x * x0.x + x0.y * x0.y;
    out[job] = make_double2(x0.x / xx, -x0.y / xx);
  }
}

cudaError_t launch_epsm(const double* re, const double* im, int neps, int nq, int nf, double2* out, cudaStream_t st) {
  if (neps > 64 || neps < 1) return cudaErrorInvalidValue;
  const int warps = 4;
  const size_t smem = (size_t)warps * neps * (neps + 1) * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(epsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int jobs = nq * nf;
  epsm_kernel<<<(jobs + warps - 1) / warps, 32 * warps, smem, st>>>(re, im, neps, nq, nf, out);
  return cudaGetLastError();
}

// Electron energy-loss function L(q, w) = -Im(1 / eps_M(q, w)) (the quantity
// the macroscopic dielectric function of macroscopic.m, :13-29 and :79, is
// taken for in EELS), and per q the loss peak: the plasmon. One warp per q:
// argmax of L over frequencies f >= fmin (ties to the lower f), then the
// vertex of the parabola through the peak and its two neighbours.
__global__ void __launch_bounds__(128) loss_kernel(const double2* __restrict__ epsm, int nq, int nf, int fmin,
                                                   double dfreq, double* __restrict__ loss,
                                                   double* __restrict__ peak) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= nq) return;
  const double2* e = epsm + (size_t)q * nf;
  double* L = loss + (size_t)q * nf;
  double best = -1.0;
  int bi = -1;
  for (int f = lane; f < nf; f += 32) {
    const double2 v = e[f];
    const double d = v.x * v.x + v.y * v.y;
    const double l = d > 0.0 ? v.y / d : 0.0;  // -Im(1/eps) = Im(eps) / |eps|^2
    L[f] = l;
    if (f >= fmin && (l > best || bi < 0)) {
      best = l;
      bi = f;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (oi >= 0 && (bi < 0 || ob > best || (ob == best && oi < bi))) {
      best = ob;
      bi = oi;
    }
  }
  __syncwarp();
  if (lane == 0) {
    double w = bi >= 0 ? bi * dfreq : 0.0, h = bi >= 0 ? best : 0.0;
    if (bi > 0 && bi + 1 < nf) {
      const double ym = L[bi - 1], y0 = L[bi], yp = L[bi + 1];
      const double den = ym - 2.0 * y0 + yp;
      if (den < 0.0) {
        const double t = 0.5 * (ym - yp) / den;  // in (-1/2, 1/2) at a strict maximum
        w = (bi + t) * dfreq;
        h = y0 - 0.25 * (ym - yp) * t;
      }
    }
    peak[2 * q] = w;
    peak[2 * q + 1] = h;
  }
}

cudaError_t launch_loss(const double2* epsm, int nq, int nf, int fmin, double dfreq, double* loss, double* peak,
                        cudaStream_t st) {
  if (nq <= 0 || nf <= 0) return cudaSuccess;
  loss_kernel<<<(nq + 3) / 4, 128, 0, st>>>(epsm, nq, nf, fmin, dfreq, loss, peak);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmx
