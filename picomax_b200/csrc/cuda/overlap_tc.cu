// Overlaps of the mixed-precision path on the tensor cores: tcgen05.mma
// kind::tf32 with split TF32 operands (hi + lo, three products), FP32
// accumulators in tensor memory, FP32 results for the mixed contraction.
//
// The overlaps of transition (k, c, v) are the moments
//   sum_p conj(c_s(p)) w(p) v_s'(loci[m][p]),  w in {1, G_p.x, G_p.y, G_p.z}
// (src/pmx_chi.cpp:501-548, src/pmx_chi_copy.cpp:493-531; the FP64 path's
// overlap_kernel in chi.cu computes the same sums one task per thread). For
// one k-point they are one complex GEMM D = A B with
//   rows of A:    (m, v, s')         A[(m,v,s')][p] = v_s'(loci[m][p]) (gathered)
//   columns of B: (c, s, w)          B[p][(c,s,w)]  = conj(c_s(p)) w(p)
// which one CTA computes for one k-point, up to four 128-row tiles at a time
// sharing each B chunk (the k+q vectors that the rows gather from staged in
// shared memory when they fit): the complex
// product as two real GEMMs with K stacked as (real parts, imaginary parts)
// in groups of 8 plane waves,
//   D_re = [A_re | A_im] [B_re ; -B_im],  D_im = [A_re | A_im] [B_im ; B_re],
// every operand split into TF32 hi + lo (x ~ hi + lo to 2^-22) and the three
// products hi.hi + hi.lo + lo.hi accumulated in FP32 in tensor memory. All
// 256 threads build the operand chunks (8 plane waves at a time, two stages;
// the next chunk's gathered values are loaded into registers while the
// current one is multiplied); one thread issues the MMAs and commits each
// chunk to its stage's mbarrier, which the producers wait on (bounded) before
// overwriting the stage. Warps 0-3 then read D (TMEM lane = row) and apply the
// polarisation and spin-orbit current tables exactly as overlap_kernel does,
// writing M32[t][3m+i][ch].
#include <cstdint>

#include "pmx_chi.hpp"
#include "pmx_common.cuh"
#include "pmx_tc.cuh"

namespace pmx {
namespace dev {

namespace {

using tc::fence_after;
using tc::fence_before;
using tc::mbar_init;
using tc::mma_commit;
using tc::smem_u32;
using tc::umma_desc;

constexpr int kTM = 128;                         // rows per tile
constexpr int kTK = 8;                           // TF32 elements per MMA K step (32 bytes)
constexpr int kTThr = 256;                       // threads per CTA
constexpr unsigned kTPolls = 1u << 26;
constexpr uint64_t kTWaitNs = 2000000000ull;     // 2 s unless the caller sets a limit
constexpr int kTABytes = kTM * kTK * 4;          // one of hi / lo: 4 KB
constexpr int kTBBytes = kOvlTcMaxN * kTK * 4;   // one of hi / lo of one of re / im: 4 KB
constexpr int kTG = 4;                           // row tiles multiplied together (share the B chunk)
constexpr int kTStage = kTG * 2 * kTABytes + 4 * kTBBytes;
constexpr int kAPer = kTM * kTK / kTThr;         // A elements per thread and chunk
constexpr int kBPer = kOvlTcMaxN * kTK / kTThr;  // B elements per thread and chunk (at most)

// x ~ hi + lo, both TF32 (round to nearest, ties away)
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  const float r = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}

// four consecutive FP32 columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float (&o)[4]) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(kTThr, 1) overlap_tc_kernel(OverlapTcArgs t, int vsm) {
  const OverlapArgs& a = t.a;
  const int k = blockIdx.x;
  const int ncd = a.ncd[k], nvd = a.nvd[k];
  const int S = a.soc ? 2 : 1;  // resolved spin components
  const int nrows = a.neps * nvd * S;
  const int nrt = (nrows + kTM - 1) / kTM;
  const int CW = kOvlTcMaxN / (4 * S);  // conduction states per column tile
  const int c_lo = blockIdx.z * CW, c_hi = min(ncd, c_lo + CW);
  if (nrows <= 0 || c_lo >= c_hi) return;
  const int ncol = 4 * S * (c_hi - c_lo);
  int N = 16;  // a power of two, so that each thread's B column is the same in every chunk
  while (N < ncol) N <<= 1;
  // row tiles per group: each takes 2 N TMEM columns (D_re, D_im)
  const int GT = min(kTG, 512 / (2 * N));
  const int ngroups = (nrt + GT - 1) / GT;
  const int kp = (a.npw + kTK - 1) / kTK * kTK;  // plane waves, padded
  const int nchunks = 2 * kp / kTK;              // per group
  // kind::tf32: D F32, A and B TF32, K-major, N >> 3, M >> 4
  const uint32_t idesc =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);
  uint32_t ncols_alloc = 32;
  while (ncols_alloc < (uint32_t)(2 * N * GT)) ncols_alloc <<= 1;

  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * kTStage);  // [2]
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 2);
  // tables of this k-point: row offsets of the conduction vectors of the
  // column tile, loci (16-bit), G (FP32), then the k+q vectors when vsm
  int* scoff = reinterpret_cast<int*>(smem + 2 * kTStage + 64);                  // [kOvlTcMaxN / 4]
  float* sg = reinterpret_cast<float*>(scoff + kOvlTcMaxN / 4);                 // [npw][3]
  short* sloc = reinterpret_cast<short*>(sg + 3 * a.npw);                       // [neps][npw]
  double2* sv = reinterpret_cast<double2*>(
      smem + 2 * kTStage + 64 + ((sizeof(int) * (kOvlTcMaxN / 4) + sizeof(float) * 3 * a.npw +
                                  sizeof(short) * (size_t)a.neps * a.npw + 15) / 16 * 16));  // [nvd][n] when vsm
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
  if (wid == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(ncols_alloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const double2* zq = a.zq + (size_t)k * a.nev * a.n;
  const double2* zk = a.zk + (size_t)k * a.nev * a.n;
  for (int i = tid; i < c_hi - c_lo; i += kTThr) scoff[i] = a.cidx[a.cbase[k] + c_lo + i] * a.n;
  for (int i = tid; i < 3 * a.npw; i += kTThr) sg[i] = (float)a.G[i];
  for (int i = tid; i < a.neps * a.npw; i += kTThr) sloc[i] = (short)a.loci[i];
  if (vsm)
    for (int idx = tid; idx < nvd * a.n; idx += kTThr) {
      const int v = idx / a.n, r = idx - v * a.n;
      sv[idx] = zq[(size_t)a.vidx[a.vbase[k] + v] * a.n + r];
    }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *s_tmem;
  const uint64_t limit = t.wait_ns > 0 ? (uint64_t)t.wait_ns : kTWaitNs;
  const int bbytes = N * kTK * 4;

  // chunk J = g * nchunks + j (group g of row tiles, chunk j of its K). This
  // thread's A elements, in each tile of the group, are row tid % 128,
  // k = tid / 128 + 2 i (i < 4); its B elements column tid % N,
  // k = tid / N + (256 / N) i (while < 8). K order: plane waves p0 .. p0 + 7,
  // real parts of A (even chunks) then imaginary parts (odd chunks), so that
  // the FP32 accumulator takes each group's Re(a) Re(b) and Im(a) Im(b) terms
  // back to back (they largely cancel in the real part).
  const int ar = tid % kTM, ak0 = tid / kTM;
  const int bcol = tid % N, bk0 = tid / N, bstep = kTThr / N;
  const bool bcol_ok = bcol < ncol;
  const int bw = bcol & 3, bs = (bcol >> 2) % S, bc = bcol / (4 * S);
  const double2* bz = zk + (bcol_ok ? scoff[bc] : 0) + bs;  // element p at bz[p * S]
  const int aoff = ((ar >> 3) * 128 + (ar & 7) * 16);       // tile offset of row ar (k group 0)
  const int boff = ((bcol >> 3) * 128 + (bcol & 7) * 16);
  // rows of this thread in the current group's tiles
  int cur_g = -1, a_sp[kTG];
  bool a_ok[kTG];
  const short* a_loc[kTG];
  const double2* a_vec[kTG];
  auto set_rows = [&](int g) {
    cur_g = g;
#pragma unroll
    for (int tt = 0; tt < kTG; ++tt) {
      const int R = (g * GT + tt) * kTM + ar;
      const bool ok = tt < GT && R < nrows;
      const int sp = ok ? R % S : 0, v = ok ? (R / S) % nvd : 0, m = ok ? R / (S * nvd) : 0;
      a_ok[tt] = ok;
      a_sp[tt] = sp;
      a_loc[tt] = sloc + m * a.npw;
      a_vec[tt] = vsm ? sv + (size_t)v * a.n : zq + (size_t)a.vidx[a.vbase[k] + v] * a.n;
    }
  };
  float av[kTG][kAPer], bre[kBPer], bim[kBPer];
  auto fetch = [&](int J) {
    const int g = J / nchunks, j = J - g * nchunks;
    if (g != cur_g) set_rows(g);
    const bool imh = (j & 1) != 0;
    const int p0 = (j >> 1) * kTK;
#pragma unroll
    for (int tt = 0; tt < kTG; ++tt)
#pragma unroll
      for (int i = 0; i < kAPer; ++i) {
        const int p = p0 + ak0 + 2 * i;
        float x = 0.f;
        if (a_ok[tt] && p < a.npw) {
          const int lp = a_loc[tt][p];
          if (lp >= 0) {
            const double2 z = a_vec[tt][S == 2 ? 2 * lp + a_sp[tt] : lp];
            x = (float)(imh ? z.y : z.x);
          }
        }
        av[tt][i] = x;
      }
#pragma unroll
    for (int i = 0; i < kBPer; ++i) {
      const int kk = bk0 + bstep * i, p = p0 + kk;
      float br = 0.f, bi = 0.f;
      if (kk < kTK && bcol_ok && p < a.npw) {
        const double2 cz = bz[(size_t)p * S];
        const double g = bw == 0 ? 1.0 : (double)sg[3 * p + bw - 1];
        // B = conj(c) g; stacked: [B_re ; -B_im] and [B_im ; B_re]
        br = (float)(imh ? cz.y * g : cz.x * g);
        bi = (float)(imh ? cz.x * g : -cz.y * g);
      }
      bre[i] = br;
      bim[i] = bi;
    }
  };

  const int A = 3 * a.neps;
  const int total = ngroups * nchunks;
  bool ok = true;
  int last = -1;  // last committed chunk
  fetch(0);
  for (int J = 0; J < total && ok; ++J) {
    const int s = J & 1, g = J / nchunks, j = J - g * nchunks;
    const int gt = min(GT, nrt - g * GT);  // tiles in this group
    uint8_t* st = smem + s * kTStage;
    // the stage is free once the MMAs of chunk J - 2 completed (one thread
    // polls, the others wait at the barrier)
    const bool fail = tid == 0 && J >= 2 && !tc::mbar_wait(&bars[s], ((J - 2) >> 1) & 1, limit, kTPolls);
    if (__syncthreads_or(fail)) {
      ok = false;
      break;
    }
#pragma unroll
    for (int tt = 0; tt < kTG; ++tt) {
      if (tt < gt) {
        uint8_t* sa = st + tt * 2 * kTABytes;
#pragma unroll
        for (int i = 0; i < kAPer; ++i) {
          const int kk = ak0 + 2 * i;
          uint32_t hi, lo;
          split_tf32(av[tt][i], hi, lo);
          const int o = aoff + (kk >> 2) * (kTM / 8) * 128 + (kk & 3) * 4;
          *reinterpret_cast<uint32_t*>(sa + o) = hi;
          *reinterpret_cast<uint32_t*>(sa + kTABytes + o) = lo;
        }
      }
    }
    uint8_t* sb = st + kTG * 2 * kTABytes;
#pragma unroll
    for (int i = 0; i < kBPer; ++i) {
      const int kk = bk0 + bstep * i;
      if (kk < kTK) {
        uint32_t h, l;
        const int o = boff + (kk >> 2) * (N / 8) * 128 + (kk & 3) * 4;
        split_tf32(bre[i], h, l);
        *reinterpret_cast<uint32_t*>(sb + o) = h;
        *reinterpret_cast<uint32_t*>(sb + bbytes + o) = l;
        split_tf32(bim[i], h, l);
        *reinterpret_cast<uint32_t*>(sb + 2 * bbytes + o) = h;
        *reinterpret_cast<uint32_t*>(sb + 3 * bbytes + o) = l;
      }
    }
    if (J + 1 < total) fetch(J + 1);  // in flight while chunk J is multiplied
    tc::async_proxy_fence();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      const uint32_t s0 = smem_u32(st), sbb = s0 + kTG * 2 * kTABytes;
      const uint32_t alb = (kTM / 8) * 128, blb = (uint32_t)(N / 8) * 128;
      const uint64_t rh = umma_desc(sbb, blb, 128), rl = umma_desc(sbb + bbytes, blb, 128);
      const uint64_t ih = umma_desc(sbb + 2 * bbytes, blb, 128), il = umma_desc(sbb + 3 * bbytes, blb, 128);
      const uint32_t acc0 = j > 0 ? 1u : 0u;  // a group's first chunk starts its accumulators
      for (int tt = 0; tt < gt; ++tt) {
        const uint32_t sa = s0 + tt * 2 * kTABytes;
        const uint64_t ahi = umma_desc(sa, alb, 128), alo = umma_desc(sa + kTABytes, alb, 128);
        const uint32_t dre = tmem + (uint32_t)(tt * 2 * N), dim = dre + N;
        mma_tf32(dre, ahi, rh, idesc, acc0);
        mma_tf32(dre, ahi, rl, idesc, 1u);
        mma_tf32(dre, alo, rh, idesc, 1u);
        mma_tf32(dim, ahi, ih, idesc, acc0);
        mma_tf32(dim, ahi, il, idesc, 1u);
        mma_tf32(dim, alo, ih, idesc, 1u);
      }
      if (!(t.fault == 4 && J == 0)) mma_commit(&bars[s]);
    }
    last = J;
    if (j != nchunks - 1) continue;
    // ---- group g complete: every MMA has completed once its last commit
    // has (bounded wait); warps 0-3 read D (TMEM lane = row) tile by tile
    const bool done = tid != 0 || tc::mbar_wait(&bars[s], (J >> 1) & 1, limit, kTPolls);
    if (__syncthreads_or(!done)) {
      ok = false;
      break;
    }
    fence_after();
    if (wid < 4) {
      for (int tt = 0; tt < gt; ++tt) {
        const int R = (g * GT + tt) * kTM + wid * 32 + lane;
        const bool row_ok = R < nrows;
        const int sp = row_ok ? R % S : 0, v = row_ok ? (R / S) % nvd : 0, m = row_ok ? R / (S * nvd) : 0;
        const double wx = (a.kpts[3 * k] + a.q[0] / 2) + a.G[3 * m] / 2;
        const double wy = (a.kpts[3 * k + 1] + a.q[1] / 2) + a.G[3 * m + 1] / 2;
        const double wz = (a.kpts[3 * k + 2] + a.q[2] / 2) + a.G[3 * m + 2] / 2;
        const uint32_t dbase = tmem + ((uint32_t)(wid * 32) << 16) + (uint32_t)(tt * 2 * N);
        for (int c = c_lo; c < c_hi; ++c) {
          // this row's moments for spin s of the conduction state: D[(c, s, w)]
          double2 mo[2][4];
          for (int s2 = 0; s2 < S; ++s2) {
            float re[4], im[4];
            const uint32_t col = (uint32_t)(((c - c_lo) * S + s2) * 4);
            tmem_ld4(dbase + col, re);
            tmem_ld4(dbase + N + col, im);
#pragma unroll
            for (int w = 0; w < 4; ++w) mo[s2][w] = make_double2(re[w], im[w]);
          }
          if (S == 2 && a.nch == 1) {
            // spin-summed: this row's own spin plus the partner row's (lane ^ 1)
#pragma unroll
            for (int w = 0; w < 4; ++w) {
              const double2 own = mo[sp][w];
              const double px = __shfl_xor_sync(0xffffffffu, own.x, 1), py = __shfl_xor_sync(0xffffffffu, own.y, 1);
              mo[0][w] = make_double2(own.x + px, own.y + py);
            }
          }
          if (!row_ok) continue;
          const long long dst = a.dest[a.blkoff[k] + (long long)c * nvd + v];
          if (dst < 0) continue;
          if (S == 2 && a.nch == 1 && sp != 0) continue;  // the pair's first row writes
          float2* out = t.M32 + ((size_t)dst * A + 3 * m) * a.nch;
          for (int i = 0; i < 3; ++i) {
            const double2* u = a.uvec + ((size_t)m * 3 + i) * 3;
            const double2 sso = a.ssoc[m * 3 + i];
            auto orb = [&](const double2* mm) {
              double2 rr = cmulc(u[0], cadd(mm[1], cscale(mm[0], wx)));
              rr = cadd(rr, cmulc(u[1], cadd(mm[2], cscale(mm[0], wy))));
              rr = cadd(rr, cmulc(u[2], cadd(mm[3], cscale(mm[0], wz))));
              return rr;
            };
            auto put = [&](int ch, double2 val) {
              out[(size_t)i * a.nch + ch] = make_float2((float)val.x, (float)val.y);
            };
            if (a.nch == 4) {
              // row s' = up: channel up (s = up) and downup (conj(c_dn) v_up);
              // row s' = down: channel down and updown (conj(c_up) v_dn)
              if (sp == 0) {
                put(0, orb(mo[0]));
                put(3, cmul(sso, mo[1][0]));
              } else {
                put(1, orb(mo[1]));
                put(2, cmul(sso, mo[0][0]));
              }
            } else {
              const double2* mm = mo[0];
              if (a.mode == 1)
                put(0, i == 0 ? mm[0] : cadd(orb(mm), cmul(sso, mm[0])));
              else
                put(0, orb(mm));
            }
          }
        }
      }
    }
    // the next group's first MMAs overwrite the accumulators
    fence_before();
    __syncthreads();
    fence_after();
  }
  if (!ok) {
    // drain: the last commit completes after every earlier MMA (bounded)
    if (tid == 0) {
      if (last >= 0) tc::mbar_wait(&bars[last & 1], (last >> 1) & 1, limit, kTPolls);
      atomicExch(t.err, 1);
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (wid == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols_alloc));
}

}  // namespace

constexpr size_t kTVsmMax = 96 * 1024;  // largest staged k+q vector block

// stages, barriers and the k-point's tables (without the staged vectors)
size_t overlap_tc_smem_bytes(int npw, int neps) {
  return (size_t)2 * kTStage + 64 +
         (sizeof(int) * (kOvlTcMaxN / 4) + sizeof(float) * 3 * npw + sizeof(short) * (size_t)neps * npw + 15) / 16 *
             16;
}

cudaError_t launch_overlap_tc(const OverlapTcArgs& t, int nk, cudaStream_t st) {
  const int S = t.a.soc ? 2 : 1;
  if (t.a.nch == 4 && S != 2) return cudaErrorInvalidValue;
  const int CW = kOvlTcMaxN / (4 * S);
  dim3 grid(nk, 1, (t.a.ncd_max + CW - 1) / CW);
  if (nk <= 0 || grid.z == 0 || t.a.nvd_max <= 0) return cudaSuccess;
  const size_t vbytes = sizeof(double2) * (size_t)t.a.nvd_max * t.a.n;
  if (t.a.npw > 32767) return cudaErrorInvalidValue;  // 16-bit loci
  const size_t base = overlap_tc_smem_bytes(t.a.npw, t.a.neps);
  const int vsm = base + vbytes <= (size_t)200 * 1024 && vbytes <= kTVsmMax ? 1 : 0;
  const size_t sm = base + (vsm ? vbytes : 0);
  if (sm > (size_t)227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(overlap_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  overlap_tc_kernel<<<grid, kTThr, sm, st>>>(t, vsm);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmx
