// Transition list of one q on the device: occupations, the distinct solved
// states of each k-point, the (k, c, v) transitions with their energies,
// weights and window starts, and a stable counting sort by window start.
//
// Occupations and transitions follow chi_tensor (src/pmx_chi.cpp:391-397,
// :477-483; conduction states counted down from the top of the NBAND window
// while E - E_ref > 0, valence states up from the bottom while <= 0), chi_LL
// (src/pmx_chi_copy.cpp, same rule) and chi_xyz (src/pmx_chi_copy.cpp:1128-1140,
// :1178-1186: valence at k, conduction at k+q). Without spin-orbit coupling
// the spatial states carry a spin multiplicity of 1 or 2 in the weight.
// Transitions are numbered in k order (pairs in (c, v) order inside a k);
// the sort by window start is stable, so the order is the one of a serial
// counting sort.
#include <algorithm>

#include "pmx_chi.hpp"

namespace pmx {
namespace dev {

namespace {

__device__ __forceinline__ double seig(const double* w, int nval, int k, int s, int soc) {
  return soc ? w[(size_t)k * nval + s] : w[(size_t)k * nval + s / 2];
}

// Occupied counts of k-point k in the NBAND window and its distinct solved
// states. The distinct states are consecutive, so they are given by index:
// conduction (first) state i and valence (second) state i.
struct KStates {
  int nc, nv;    // occupied counts in the window (spinor states)
  int ncd, nvd;  // distinct solved states
  int nband, soc, xyz;
  __device__ int cs(int i) const {
    if (xyz) return i;                            // valence at k, counted up
    return soc ? nband - 1 - i : (nband - 1) / 2 - i;  // (nband - 1 - c) / 2 for c = 0, 1, ...
  }
  __device__ int vs(int i) const {
    if (xyz) return nband - 1 - i;                // conduction at k+q, counted down
    return i;                                     // v (SOC) or v / 2 for v = 0, 1, ...
  }
};

__device__ void k_states(const TransArgs& a, int k, KStates& S) {
  const int NB = a.nband, soc = a.soc;
  int nc = 0, nv = 0;
  if (a.xyz) {
    while (nc < NB && seig(a.wk, a.nval, k, nc, soc) - a.off <= 0) ++nc;
    while (nv < NB && seig(a.wq, a.nval, k, NB - 1 - nv, soc) - a.off > 0) ++nv;
  } else {
    while (nc < NB && seig(a.wk, a.nval, k, NB - 1 - nc, soc) - a.off > 0) ++nc;
    while (nv < NB && seig(a.wq, a.nval, k, nv, soc) - a.off <= 0) ++nv;
  }
  S.nc = nc;
  S.nv = nv;
  S.nband = NB;
  S.soc = soc;
  S.xyz = a.xyz;
  if (a.xyz || soc) {
    S.ncd = nc;
    S.nvd = nv;
  } else {
    S.ncd = nc > 0 ? (NB - 1) / 2 - (NB - nc) / 2 + 1 : 0;
    S.nvd = nv > 0 ? (nv - 1) / 2 + 1 : 0;
  }
}

__device__ __forceinline__ int pair_mult(const TransArgs& a, const KStates& S, int ic, int iv) {
  if (a.xyz || a.soc) return 1;
  const int NB = a.nband;
  int mult = 0;
  for (int sg = 0; sg < 2; ++sg) {
    const int sc = 2 * S.cs(ic) + sg, sv = 2 * S.vs(iv) + sg;
    const int c = NB - 1 - sc;
    if (sc <= NB - 1 && c >= 0 && c < S.nc && sv < S.nv) ++mult;
  }
  return mult;
}

__device__ __forceinline__ double pair_de(const TransArgs& a, const KStates& S, int k, int ic, int iv) {
  if (a.xyz)
    return (seig(a.wq, a.nval, k, S.vs(iv), a.soc) - a.off) - (seig(a.wk, a.nval, k, S.cs(ic), a.soc) - a.off);
  const int s_c = a.soc ? S.cs(ic) : 2 * S.cs(ic);
  const int s_v = a.soc ? S.vs(iv) : 2 * S.vs(iv);
  const double ec = seig(a.wk, a.nval, k, s_c, a.soc) - a.off;
  const double ev = seig(a.wq, a.nval, k, s_v, a.soc) - a.off;
  return ec - ev;
}

__global__ void trans_occ_kernel(TransArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nk) return;
  const int NB = a.nband, soc = a.soc;
  int cuts = 0, ties = 0;
  if (NB < a.nh) {
    cuts += fabs(seig(a.wk, a.nval, k, NB, soc) - seig(a.wk, a.nval, k, NB - 1, soc)) < 1e-8 ? 1 : 0;
    cuts += fabs(seig(a.wq, a.nval, k, NB, soc) - seig(a.wq, a.nval, k, NB - 1, soc)) < 1e-8 ? 1 : 0;
  }
  {
    bool tk = false, tq = false;
    for (int s = 0; s < NB && s < a.nh; ++s) {
      tk |= fabs(seig(a.wk, a.nval, k, s, soc) - a.off) < 1e-8;
      tq |= fabs(seig(a.wq, a.nval, k, s, soc) - a.off) < 1e-8;
    }
    ties = (int)tk + (int)tq;
  }
  KStates S;
  k_states(a, k, S);
  int ntr = 0, lo = INT_MAX, hi = INT_MIN;
  for (int ic = 0; ic < S.ncd; ++ic)
    for (int iv = 0; iv < S.nvd; ++iv) {
      if (pair_mult(a, S, ic, iv) == 0) continue;
      const int f0 = (int)((pair_de(a, S, k, ic, iv) - a.w0) / a.df);
      lo = min(lo, f0);
      hi = max(hi, f0);
      ++ntr;
    }
  a.ncd[k] = S.ncd;
  a.nvd[k] = S.nvd;
  a.cbase[k] = k * NB;
  a.vbase[k] = k * NB;
  for (int i = 0; i < S.ncd; ++i) a.cidx[(size_t)k * NB + i] = S.cs(i);
  for (int i = 0; i < S.nvd; ++i) a.vidx[(size_t)k * NB + i] = S.vs(i);
  a.ntr[k] = ntr;
  a.nblk[k] = S.ncd * S.nvd;
  if (cuts) atomicAdd(&a.sum->cuts, cuts);
  if (ties) atomicAdd(&a.sum->ties, ties);
  if (ntr) {
    atomicMin(&a.sum->f0_lo, lo);
    atomicMax(&a.sum->f0_hi, hi);
  }
  atomicMax(&a.sum->ncd_max, S.ncd);
  atomicMax(&a.sum->nvd_max, S.nvd);
}

// One CTA: exclusive scans of the per-k block sizes and transition counts.
__global__ void trans_scan_kernel(TransArgs a) {
  __shared__ long long ws1[32], ws2[32];
  __shared__ long long base1, base2;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base1 = base2 = 0;
  __syncthreads();
  for (int c0 = 0; c0 < a.nk; c0 += blockDim.x) {
    const int k = c0 + threadIdx.x;
    const long long f1 = k < a.nk ? a.nblk[k] : 0, f2 = k < a.nk ? a.ntr[k] : 0;
    long long x1 = f1, x2 = f2;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y1 = __shfl_up_sync(0xffffffffu, x1, o), y2 = __shfl_up_sync(0xffffffffu, x2, o);
      if (lane >= o) {
        x1 += y1;
        x2 += y2;
      }
    }
    if (lane == 31) {
      ws1[wid] = x1;
      ws2[wid] = x2;
    }
    __syncthreads();
    if (wid == 0) {
      long long s1 = lane < nw ? ws1[lane] : 0, s2 = lane < nw ? ws2[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y1 = __shfl_up_sync(0xffffffffu, s1, o), y2 = __shfl_up_sync(0xffffffffu, s2, o);
        if (lane >= o) {
          s1 += y1;
          s2 += y2;
        }
      }
      if (lane < nw) {
        ws1[lane] = s1;
        ws2[lane] = s2;
      }
    }
    __syncthreads();
    if (k < a.nk) {
      a.blkoff[k] = base1 + x1 - f1 + (wid > 0 ? ws1[wid - 1] : 0);
      a.toff[k] = base2 + x2 - f2 + (wid > 0 ? ws2[wid - 1] : 0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      base1 += ws1[nw - 1];
      base2 += ws2[nw - 1];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.sum->nblk = base1;
    a.sum->T = base2;
  }
}

// The transitions of each k in order, at toff[k].
__global__ void trans_fill_kernel(TransArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nk) return;
  KStates S;
  k_states(a, k, S);
  long long t = a.toff[k];
  for (int ic = 0; ic < S.ncd; ++ic)
    for (int iv = 0; iv < S.nvd; ++iv) {
      const int mult = pair_mult(a, S, ic, iv);
      if (mult == 0) continue;
      const double de = pair_de(a, S, k, ic, iv);
      a.rsrc[t] = a.blkoff[k] + (long long)ic * S.nvd + iv;
      a.rde[t] = de;
      a.rw[t] = a.kw[k] * mult;
      a.rf0[t] = (int)((de - a.w0) / a.df);
      ++t;
    }
}

// per sort block (sb transitions) and bucket: count
__global__ void trans_hist_kernel(TransArgs a, long long T, int lo, int nb, long long sb) {
  const long long t0 = (long long)blockIdx.x * sb, t1 = min(T, t0 + sb);
  for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x)
    atomicAdd(&a.cnt[(size_t)blockIdx.x * nb + (a.rf0[t] - lo)], 1);
}

// per bucket: exclusive scan over the blocks, bucket totals
__global__ void trans_bucket_kernel(TransArgs a, int nblocks, int nb) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int acc = 0;
  for (int j = 0; j < nblocks; ++j) {
    const int c = a.cnt[(size_t)j * nb + b];
    a.cnt[(size_t)j * nb + b] = acc;
    acc += c;
  }
  a.btot[b] = acc;
}

// one CTA: exclusive scan of the bucket totals -> bucket starts
__global__ void trans_bstart_kernel(TransArgs a, int nb) {
  __shared__ int ws[32];
  __shared__ int base;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < nb; c0 += blockDim.x) {
    const int b = c0 + threadIdx.x;
    const int f = b < nb ? a.btot[b] : 0;
    int x = f;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int s = lane < nw ? ws[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      if (lane < nw) ws[lane] = s;
    }
    __syncthreads();
    if (b < nb) a.btot[b] = base + x - f + (wid > 0 ? ws[wid - 1] : 0);
    __syncthreads();
    if (threadIdx.x == 0) base += ws[nw - 1];
    __syncthreads();
  }
}

// one warp per sort block, its transitions in order, 32 at a time: the lanes
// of a bucket take consecutive slots after the block's earlier ones
__global__ void trans_place_kernel(TransArgs a, long long T, int lo, int nb, long long sb) {
  const int lane = threadIdx.x;
  const long long t0 = (long long)blockIdx.x * sb, t1 = min(T, t0 + sb);
  int* pos = a.cnt + (size_t)blockIdx.x * nb;
  for (long long g = t0; g < t1; g += 32) {
    const long long t = g + lane;
    const bool in = t < t1;
    const int key = in ? a.rf0[t] - lo : -1 - lane;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const unsigned below = peers & ((1u << lane) - 1u);
    if (in) {
      const long long dst = (long long)a.btot[key] + pos[key] + __popc(below);
      a.dest[a.rsrc[t]] = dst;
      a.de[dst] = a.rde[t];
      a.wgt[dst] = a.rw[t];
      a.f0[dst] = a.rf0[t];
    }
    __syncwarp();
    if (in && below == 0) pos[key] += __popc(peers);
    __syncwarp();
  }
}

// unsorted: transition t stays at t
__global__ void trans_copy_kernel(TransArgs a, long long T) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  a.dest[a.rsrc[t]] = t;
  a.de[t] = a.rde[t];
  a.wgt[t] = a.rw[t];
  a.f0[t] = a.rf0[t];
}

// transition range of every frequency tile (sorted list: window overlap)
__global__ void trans_range_kernel(TransArgs a, long long T, int nft, int ftile, int nf, int window) {
  const int ft = blockIdx.x * blockDim.x + threadIdx.x;
  if (ft >= nft) return;
  if (window < 0) {
    a.trange[ft] = make_int2(0, (int)T);
    return;
  }
  const int flo = ft * ftile, fhi = min(nf, flo + ftile) - 1;
  // lower_bound(flo - window), upper_bound(fhi + window)
  long long l = 0, h = T;
  while (l < h) {
    const long long m = (l + h) >> 1;
    if (a.f0[m] < flo - window) l = m + 1; else h = m;
  }
  const long long b = l;
  l = 0;
  h = T;
  while (l < h) {
    const long long m = (l + h) >> 1;
    if (a.f0[m] <= fhi + window) l = m + 1; else h = m;
  }
  a.trange[ft] = make_int2((int)b, (int)l);
}

}  // namespace

cudaError_t launch_transitions_count(const TransArgs& a, cudaStream_t st) {
  if (a.nband > kTransMaxNB || a.nk <= 0) return cudaErrorInvalidValue;
  TransSummary init{};
  init.f0_lo = INT_MAX;
  init.f0_hi = INT_MIN;
  cudaError_t e = cudaMemcpyAsync(a.sum, &init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  trans_occ_kernel<<<(a.nk + 127) / 128, 128, 0, st>>>(a);
  trans_scan_kernel<<<1, 1024, 0, st>>>(a);
  return cudaGetLastError();
}

// sort blocks: at most kSortCells / nb of them (their counts fit the scratch)
constexpr long long kSortCells = 1LL << 25;
static void sort_blocks(const TransSummary& s, long long& nblocks, long long& sb) {
  const long long nb = (long long)s.f0_hi - s.f0_lo + 1;
  nblocks = std::max<long long>(1, std::min<long long>((s.T + 1023) / 1024, kSortCells / nb));
  sb = (s.T + nblocks - 1) / nblocks;
  sb = (sb + 31) / 32 * 32;
  nblocks = (s.T + sb - 1) / sb;
}

cudaError_t launch_transitions_fill(const TransArgs& a, const TransSummary& s, bool sort, int nft, int ftile, int nf,
                                    int window, cudaStream_t st) {
  const long long T = s.T;
  cudaError_t e = cudaMemsetAsync(a.dest, 0xff, sizeof(long long) * std::max<long long>(s.nblk, 1), st);
  if (e != cudaSuccess) return e;
  if (T > 0) {
    trans_fill_kernel<<<(a.nk + 127) / 128, 128, 0, st>>>(a);
    if (sort) {
      const int nb = s.f0_hi - s.f0_lo + 1;
      long long nblocks, sb;
      sort_blocks(s, nblocks, sb);
      e = cudaMemsetAsync(a.cnt, 0, sizeof(int) * (size_t)nblocks * nb, st);
      if (e != cudaSuccess) return e;
      trans_hist_kernel<<<(int)nblocks, 1024, 0, st>>>(a, T, s.f0_lo, nb, sb);
      trans_bucket_kernel<<<(nb + 255) / 256, 256, 0, st>>>(a, (int)nblocks, nb);
      trans_bstart_kernel<<<1, 1024, 0, st>>>(a, nb);
      trans_place_kernel<<<(int)nblocks, 32, 0, st>>>(a, T, s.f0_lo, nb, sb);
    } else {
      trans_copy_kernel<<<(int)((T + 255) / 256), 256, 0, st>>>(a, T);
    }
  }
  if (nft > 0) trans_range_kernel<<<(nft + 127) / 128, 128, 0, st>>>(a, T, nft, ftile, nf, window);
  return cudaGetLastError();
}

size_t transitions_sort_ints(const TransSummary& s) {
  if (s.T <= 0) return 1;
  const long long nb = (long long)s.f0_hi - s.f0_lo + 1;
  long long nblocks, sb;
  sort_blocks(s, nblocks, sb);
  return (size_t)(nblocks * nb + nb);
}

bool transitions_sortable(const TransSummary& s) {
  return s.T <= 0 || ((long long)s.f0_hi - s.f0_lo + 1 <= kSortCells && s.T < (1LL << 31));
}

}  // namespace dev
}  // namespace pmx
