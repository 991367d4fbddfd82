// Symmetry reduction of a Gamma-centred k-point grid on the device.
//
// The reference reads irreducible k-point lists with weights from files
// (import_kpt, src/pmx_basis.cpp:200-245; the files in include/kpoints/autoGR
// and include/kpoints/kpLib come from outside tools) and generates only full
// grids itself (src/pmx_basis.cpp:256-650). Here the irreducible wedge of the
// grid k = sum_j i_j / n_j b_j under a group of operations (integer matrices
// in the reciprocal basis, from symmetry_ops on the host) is found on the
// device: every grid point takes the smallest linear index of its orbit as
// its representative, the orbit sizes are counted, and one CTA compacts the
// representatives in index order.
#include <algorithm>

#include "pmx_device.hpp"

namespace pmx {
namespace dev {

namespace {

__device__ __forceinline__ long long pmod(long long v, int n) {
  const long long r = v % n;
  return r < 0 ? r + n : r;
}

__global__ void kgrid_rep_kernel(KgridOps ops, int n1, int n2, int n3, int* __restrict__ rep, int* __restrict__ cnt) {
  const long long N = (long long)n1 * n2 * n3;
  for (long long L = (long long)blockIdx.x * blockDim.x + threadIdx.x; L < N; L += (long long)gridDim.x * blockDim.x) {
    const long long i1 = L % n1, i2 = (L / n1) % n2, i3 = L / ((long long)n1 * n2);
    long long best = L;
    for (int o = 0; o < ops.n; ++o) {
      const int* M = ops.m[o];
      const long long j1 = pmod(M[0] * i1 + M[1] * i2 + M[2] * i3, n1);
      const long long j2 = pmod(M[3] * i1 + M[4] * i2 + M[5] * i3, n2);
      const long long j3 = pmod(M[6] * i1 + M[7] * i2 + M[8] * i3, n3);
      const long long J = j1 + (long long)n1 * (j2 + (long long)n2 * j3);
      best = J < best ? J : best;
    }
    rep[L] = (int)best;
    atomicAdd(&cnt[best], 1);
  }
}

// One CTA: block-wide exclusive scans of the representative flags, chunk by
// chunk, so that the output is in grid-index order.
__global__ void kgrid_compact_kernel(const int* __restrict__ rep, const int* __restrict__ cnt, int n1, int n2,
                                     long long N, int* __restrict__ idx, int* __restrict__ w, int* __restrict__ nirr) {
  __shared__ int wsum[32];
  __shared__ int base;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (long long c0 = 0; c0 < N; c0 += blockDim.x) {
    const long long L = c0 + threadIdx.x;
    const int f = (L < N && rep[L] == L) ? 1 : 0;
    int x = f;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int s = lane < nw ? wsum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      if (lane < nw) wsum[lane] = s;
    }
    __syncthreads();
    const int pos = base + x - f + (wid > 0 ? wsum[wid - 1] : 0);
    if (f && idx) {
      idx[3 * (size_t)pos] = (int)(L % n1);
      idx[3 * (size_t)pos + 1] = (int)((L / n1) % n2);
      idx[3 * (size_t)pos + 2] = (int)(L / ((long long)n1 * n2));
      w[pos] = cnt[L];
    }
    __syncthreads();
    if (threadIdx.x == 0) base += wsum[nw - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *nirr = base;
}

}  // namespace

cudaError_t launch_kgrid_reduce(const KgridOps& ops, const int* n, int* rep, int* cnt, int* idx, int* w, int* nirr,
                                cudaStream_t st) {
  const long long N = (long long)n[0] * n[1] * n[2];
  if (N <= 0 || N > (1LL << 30) || ops.n < 1 || ops.n > kKgridMaxOps) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int) * N, st);
  if (e != cudaSuccess) return e;
  const int threads = 256;
  const long long blocks = std::min<long long>((N + threads - 1) / threads, 148LL * 16);
  kgrid_rep_kernel<<<(int)blocks, threads, 0, st>>>(ops, n[0], n[1], n[2], rep, cnt);
  kgrid_compact_kernel<<<1, 1024, 0, st>>>(rep, cnt, n[0], n[1], N, idx, w, nirr);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmx
