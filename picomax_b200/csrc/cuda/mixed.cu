// Mixed-precision chi contraction on the sm_100a tensor cores.
//
// The contraction acc[p, f] = sum_t P[p, t] W[t, f] of the FP64 path (pair
// products P of the overlaps, broadening weights W inside each transition's
// window) runs as a GEMM with
//   rows  = 64 (a, b) pairs x {P1 = w reO, P2 = -w imO}      (M = 128)
//   cols  = 256 frequencies                                 (N = 256)
//   depth = transitions of the frequency tile, 32 per chunk (K)
// Operands are split into BF16 pairs, x = hi + lo, and every chunk issues
// hi*hi + hi*lo + lo*hi as tcgen05.mma kind::f16 with an FP32 accumulator in
// TMEM (products dropped: lo*lo, ~2^-16 of each term). The transition range
// of a frequency tile is cut into pieces; each piece adds its FP32
// accumulator into an FP64 partial tile every 64 chunks, and the pieces'
// tiles are summed in FP64 in a fixed order, so results are deterministic.
//
// Pipeline of one CTA (8 producer warps + 1 control warp, two shared-memory
// stages):
//   control    bulk-copies the precomputed W chunk (hi and lo, 32 KB, already
//              in the canonical K-major UMMA layout) into a stage once the
//              stage's previous MMAs completed; waits for the stage's A tile
//              and W copy, issues 6 MMAs and commits them to the stage's
//              mbarrier
//   producers  stage the overlaps of the chunk in shared memory (named
//              barrier among the producers only), write the split P tile and
//              arrive on the stage's A-full mbarrier; warps 0-3 move the FP32
//              accumulator to the FP64 tile after every 64 chunks.
// Every mbarrier wait is bounded; on expiry the CTA records an error code,
// drains its own MMAs and W copies (bounded), frees its TMEM and returns. The producers
// leave their loop together: the decision is an OR over a named barrier.
#include <cuda_bf16.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>

#include "pmx_common.cuh"
#include "pmx_mixed.hpp"
#include "pmx_tc.cuh"

namespace pmx {
namespace dev {

namespace {

constexpr int kM = 128;        // MMA rows
constexpr int kPairs = 64;     // pairs per tile (kM / 2)
constexpr int kN = 256;        // frequencies per tile
constexpr int kKC = 32;        // transitions per chunk
constexpr int kProducers = 256;              // warps 0-7
constexpr int kThreads = kProducers + 32;    // + the control warp (W copies, MMA issue)
constexpr int kFlushChunks = 64;  // chunks (2048 transitions) per FP32 accumulation before the FP64 flush
constexpr int kTargetCtas = 4 * 148;  // K-split so that the grid covers the SMs a few times
constexpr unsigned kWaitLimit = 1u << 26;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s, unless the caller sets a limit

// canonical K-major, no-swizzle layout: core matrices of 8 rows x 16 bytes;
// rows of a core matrix 16 B apart, row groups SBO = 128 B apart, 8-element
// K chunks LBO = rows/8 * 128 B apart.
constexpr int kABytes = kM * kKC * 2;  // one of hi/lo: 8 KB
constexpr int kBBytes = kN * kKC * 2;  // one of hi/lo: 16 KB
constexpr int kWChunkBytes = 2 * kBBytes;  // hi + lo in global and in the stage

__host__ __device__ constexpr int core_off(int r, int k, int rows) {
  return ((k >> 3) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

using tc::global_ns;
using tc::mbar_arrive;
using tc::mbar_init;
using tc::mma_commit;
using tc::smem_u32;
using tc::umma_desc;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  return tc::mbar_wait(bar, parity, limit_ns, kWaitLimit);
}
__device__ __forceinline__ void tc_fence_after() { tc::fence_after(); }
__device__ __forceinline__ void tc_fence_before() { tc::fence_before(); }
__device__ __forceinline__ void async_proxy_fence() { tc::async_proxy_fence(); }

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, A and B K-major.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kM >> 4) << 24);

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(acc)
      : "memory");
}

// Named barrier 1 over the producer warps, returning the OR of v over them
// (every producer gets the same answer).
__device__ __forceinline__ bool producers_sync_or(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, 1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "n"(kProducers)
      : "memory");
  return r != 0;
}

// hi/lo split of 8 values into two 16-byte rows of a core matrix:
// hi = bf16_rn(x), lo = bf16_rn(x - hi), two values per conversion.
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
    const float2 hf = __bfloat1622float2(hb);
    const __nv_bfloat162 lb = __floats2bfloat162_rn(x[2 * i] - hf.x, x[2 * i + 1] - hf.y);
    h[i] = *reinterpret_cast<const uint32_t*>(&hb);
    l[i] = *reinterpret_cast<const uint32_t*>(&lb);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ double broaden_m(int model, double eps, double x) {
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

// ------------------------------------------------------------- work plan
struct Plan {
  int nft;           // frequency tiles
  int ntile;         // pair tiles
  int nchunk;        // W chunks over all frequency tiles
  int nitem;         // (frequency tile, piece) items
  // device arrays inside the workspace
  int* chunk_ft;     // [nchunk] frequency tile of the chunk
  int* chunk_t0;     // [nchunk] first sorted transition of the chunk
  int* chunk_t1;     // [nchunk] end of the frequency tile's range
  int4* item;        // [nitem] (ft, first chunk, end chunk, -)
  int2* ft_items;    // [nft] (first item, end item)
  int2* tiles;       // [ntile] (a block, b block)
  float* wgt32;      // [T]
  uint8_t* wbuf;     // [nchunk][32 KB]
  double* part;      // [nitem][ntile] FP64 partial tiles of 128 x 256, see part_index
  int* err;          // error flag
  uint64_t wait_ns;  // limit of every bounded wait
  int fault;         // tests only: 1 = the producers withhold their first A-full arrival
};

// Layout of a 128 x 256 partial tile: four 32-row blocks (one per TMEM lane
// quarter), each column-major: a flush pass of one warp (32 rows x 32
// columns) is one contiguous 8 KB block.
__host__ __device__ constexpr int part_index(int row, int col) { return (row >> 5) * (kN * 32) + col * 32 + (row & 31); }

__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes, bool add) {
  if (add)
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;" ::"l"(gdst),
                 "r"(smem_u32(ssrc)), "r"(bytes)
                 : "memory");
  else
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(ssrc)),
                 "r"(bytes)
                 : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace

// -------------------------------------------------------- W chunk producer
__global__ void __launch_bounds__(256) wgen_kernel(Plan pl, ContractArgs a) {
  const int c = blockIdx.x;
  const int ft = pl.chunk_ft[c], t0 = pl.chunk_t0[c], t1 = pl.chunk_t1[c];
  uint8_t* out = pl.wbuf + (size_t)c * kWChunkBytes;
  // each thread writes 16-byte rows: (freq n, k-group kg) -> 8 transitions
  for (int idx = threadIdx.x; idx < kN * (kKC / 8); idx += blockDim.x) {
    const int n = idx % kN, kg = idx / kN;
    const int f = ft * kN + n;
    float x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int t = t0 + kg * 8 + q;
      double v = 0.0;
      if (t < t1 && f < a.nf) {
        const bool in = a.window < 0 || abs(f - a.f0[t]) <= a.window;
        if (in) v = broaden_m(a.delta, a.eps, a.dE[t] - a.dfreq * f);
      }
      x[q] = (float)v;
    }
    uint4 hi, lo;
    split8(x, hi, lo);
    const int off = core_off(n, kg * 8, kN);
    *reinterpret_cast<uint4*>(out + off) = hi;
    *reinterpret_cast<uint4*>(out + kBBytes + off) = lo;
  }
}

// ------------------------------------------------------------- main GEMM
template <int NCH>
__global__ void __launch_bounds__(kThreads, 2) mixed_kernel(Plan pl, ContractArgs a, const float2* __restrict__ M32) {
  const int tile = blockIdx.x, item_id = blockIdx.y;
  const int2 tb = pl.tiles[tile];
  const int4 it = pl.item[item_id];
  const int c_begin = it.y, nch = it.z - it.y;
  const int A = 3 * a.neps;
  const int a0 = tb.x * 8, b0 = tb.y * 8;
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
  // the chunks of an item are consecutive 32-transition slices of one
  // frequency tile's range
  const int t_first = nch > 0 ? pl.chunk_t0[c_begin] : 0, t_end = nch > 0 ? pl.chunk_t1[c_begin] : 0;

  // overlaps staged per chunk: double-buffered when small (NCH = 1), so that
  // one producer barrier per chunk suffices
  constexpr int kSMBuf = NCH == 1 ? 2 : 1;
  // staged overlaps: 16 slot rows (8 a-side, 8 b-side) of kKC transitions x
  // NCH, each row padded by 16 bytes so that the producers' 16-byte reads of
  // 8 different b-rows by a quarter warp fall into distinct banks
  constexpr int kRow = kKC * NCH + 2;
  constexpr int kSMElems = 16 * kRow;
  extern __shared__ __align__(1024) uint8_t smem[];
  // stage layout: [A hi 8K][A lo 8K][B hi 16K][B lo 16K] x 2
  auto stage = [&](int s) { return smem + s * (2 * kABytes + kWChunkBytes); };
  float2* sM = reinterpret_cast<float2*>(smem + 2 * (2 * kABytes + kWChunkBytes));  // [kSMBuf][16][kRow]
  float* sw = reinterpret_cast<float*>(sM + kSMBuf * kSMElems);                      // [kSMBuf][kKC]
  uint64_t* bars = reinterpret_cast<uint64_t*>(sw + kSMBuf * kKC);  // wfull[2], mdone[2], afull[2]
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 6);
  int* s_abort = reinterpret_cast<int*>(s_tmem + 1);  // s_abort[0], last committed chunk s_abort[1]
  int* s_last = s_abort + 1;
  uint64_t* wfull = bars;
  uint64_t* mdone = bars + 2;
  uint64_t* afull = bars + 4;

  if (wid == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(kN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < 4; ++i) mbar_init(&bars[i], 1);
    for (int i = 4; i < 6; ++i) mbar_init(&bars[i], kProducers);
    *s_abort = 0;
    *s_last = -1;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  // a bounded wait that gives up at once when the CTA already aborted
  auto wait = [&](uint64_t* bar, uint32_t parity, int code) {
    if (*(volatile int*)s_abort) return false;
    if (mbar_wait(bar, parity, pl.wait_ns)) return true;
    atomicExch(pl.err, code);
    *(volatile int*)s_abort = 1;
    return false;
  };

  if (wid == kProducers / 32) {
    // ------------------------------------------------------------ control
    if (lane == 0) {
      // W chunks whose bulk copy was issued / has landed: on an abort the
      // copies still in flight are waited for before the CTA frees anything
      int issued = -1, landed = -1;
      for (int n = 0; n < 2 && n < nch; ++n) {
        bulk_load(stage(n) + 2 * kABytes, pl.wbuf + (size_t)(c_begin + n) * kWChunkBytes, kWChunkBytes, &wfull[n]);
        issued = n;
      }
      for (int n = 0; n < nch; ++n) {
        const int s = n & 1, g = n % kFlushChunks;
        if (!wait(&afull[s], (n >> 1) & 1, 5) || !wait(&wfull[s], (n >> 1) & 1, 2)) break;
        landed = n;
        tc_fence_after();
        const uint32_t sa = smem_u32(stage(s));
        const uint32_t sb = sa + 2 * kABytes;
#pragma unroll
        for (int ks = 0; ks < kKC / 16; ++ks) {
          // K step ks covers k-groups 2ks, 2ks+1: +2*LBO bytes
          const uint64_t ahi = umma_desc(sa + ks * 2 * (kM / 8) * 128, (kM / 8) * 128, 128);
          const uint64_t alo = umma_desc(sa + kABytes + ks * 2 * (kM / 8) * 128, (kM / 8) * 128, 128);
          const uint64_t bhi = umma_desc(sb + ks * 2 * (kN / 8) * 128, (kN / 8) * 128, 128);
          const uint64_t blo = umma_desc(sb + kBBytes + ks * 2 * (kN / 8) * 128, (kN / 8) * 128, 128);
          const uint32_t acc0 = (g > 0 || ks > 0) ? 1u : 0u;
          mma_bf16(tmem, ahi, bhi, acc0);
          mma_bf16(tmem, ahi, blo, 1u);
          mma_bf16(tmem, alo, bhi, 1u);
        }
        mma_commit(&mdone[s]);
        *(volatile int*)s_last = n;
        // the other stage is free once chunk n-1's MMAs (queued ahead of
        // chunk n's) completed: its W copy for chunk n+1 starts then
        if (n >= 1 && n + 1 < nch) {
          if (!wait(&mdone[s ^ 1], ((n - 1) >> 1) & 1, 1)) break;
          bulk_load(stage(s ^ 1) + 2 * kABytes, pl.wbuf + (size_t)(c_begin + n + 1) * kWChunkBytes, kWChunkBytes,
                    &wfull[s ^ 1]);
          issued = n + 1;
        }
      }
      // drain (after an abort): every issued W copy lands before the stages
      // are released; chunk c completes phase (c >> 1) & 1 of wfull[c & 1]
      for (int c = landed + 1; c <= issued; ++c)
        if (!mbar_wait(&wfull[c & 1], (c >> 1) & 1, pl.wait_ns)) {
          atomicExch(pl.err, 6);
          break;
        }
    }
    __syncwarp();
  } else {
    // ---------------------------------------------------------- producers
    // pair handled by this thread: 64 pairs x 4 groups of 8 transitions; a
    // warp shares the a-side row, a quarter warp the transition group
    const int ia = wid, ib = tid & 7, kg = (tid >> 3) & 3;
    const int pp = ia * 8 + ib;
    const int av = a0 + ia, bv = b0 + ib;
    const bool valid = av < A && bv < A && (av / 3) >= (bv / 3);
    double* out = pl.part + ((size_t)item_id * pl.ntile + tile) * (kM * kN);
    int flushes = 0;
    // The overlaps and weights of chunk n + 1 are loaded into registers while
    // chunk n is produced, so the L2 latency of the overlap gather is off the
    // producers' critical path.
    constexpr int kMPer = kKC * 16 * NCH / kProducers;
    float2 mreg[kMPer];
    float wreg = 0.f;
    auto load_chunk = [&](int n) {
      const int t0 = t_first + n * kKC;
#pragma unroll
      for (int q = 0; q < kMPer; ++q) {
        const int idx = tid + q * kProducers;
        const int t = idx / (16 * NCH), rem = idx % (16 * NCH);
        const int slot = rem / NCH, ch = rem % NCH;
        const int gt = t0 + t;
        const int ab = slot < 8 ? a0 + slot : b0 + slot - 8;
        mreg[q] = (gt < t_end && ab < A) ? M32[((size_t)gt * A + ab) * NCH + ch] : make_float2(0.f, 0.f);
      }
      wreg = (tid < kKC && t0 + tid < t_end) ? pl.wgt32[t0 + tid] : 0.f;
    };
    if (nch > 0) load_chunk(0);
    for (int n = 0; n < nch; ++n) {
      const int s = n & 1, g = n % kFlushChunks, sb = kSMBuf == 2 ? s : 0;
      uint8_t* st = stage(s);
      float2* sMb = sM + sb * kSMElems;
      float* swb = sw + sb * kKC;
      // the stage is free once the MMAs of chunk n-2 completed
      bool fail = n >= 2 && !wait(&mdone[s], ((n - 2) >> 1) & 1, 1);
      // with one overlap buffer, every producer has finished reading chunk
      // n-1's overlaps before any overwrites them
      if (kSMBuf == 1 && producers_sync_or(fail)) break;
#pragma unroll
      for (int q = 0; q < kMPer; ++q) {
        const int idx = tid + q * kProducers;
        const int t = idx / (16 * NCH), rem = idx % (16 * NCH);
        sMb[(rem / NCH) * kRow + t * NCH + rem % NCH] = mreg[q];
      }
      if (tid < kKC) swb[tid] = wreg;
      fail = fail || *(volatile int*)s_abort;
      if (producers_sync_or(fail)) break;
      if (n + 1 < nch) load_chunk(n + 1);
      // split pair products into the A tile: row pp (P1) and 64 + pp (P2)
      {
        float p1[8], p2[8];
        // this thread's 8 transitions are contiguous in both rows: 16-byte
        // loads (all 8 up front for NCH = 1, per transition for NCH = 4)
        const float4* pa = reinterpret_cast<const float4*>(sMb + ia * kRow + kg * 8 * NCH);
        const float4* pb = reinterpret_cast<const float4*>(sMb + (8 + ib) * kRow + kg * 8 * NCH);
        float4 a1[NCH == 1 ? 4 : 1], b1[NCH == 1 ? 4 : 1];
        if (NCH == 1) {
#pragma unroll
          for (int i = 0; i < (NCH == 1 ? 4 : 1); ++i) {
            a1[i] = pa[i];
            b1[i] = pb[i];
          }
        }
        float w8[8];
        {
          const float4* pw = reinterpret_cast<const float4*>(swb + kg * 8);
          const float4 w0 = pw[0], w1 = pw[1];
          w8[0] = w0.x; w8[1] = w0.y; w8[2] = w0.z; w8[3] = w0.w;
          w8[4] = w1.x; w8[5] = w1.y; w8[6] = w1.z; w8[7] = w1.w;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          float reO = 0.f, imO = 0.f;
          if (valid) {
            if (NCH == 1) {
              const float4 va = a1[(q >> 1) & (NCH == 1 ? 3 : 0)], vb = b1[(q >> 1) & (NCH == 1 ? 3 : 0)];
              const float2 a = (q & 1) ? make_float2(va.z, va.w) : make_float2(va.x, va.y);
              const float2 b = (q & 1) ? make_float2(vb.z, vb.w) : make_float2(vb.x, vb.y);
              reO = a.x * b.x + a.y * b.y;
              imO = a.y * b.x - a.x * b.y;
            } else {
              // channels up, dn, ud, du of transition q: 2 x 16 bytes per row
              const float4 a01 = pa[2 * q], a23 = pa[2 * q + 1], b01 = pb[2 * q], b23 = pb[2 * q + 1];
              const float2 a[4] = {make_float2(a01.x, a01.y), make_float2(a01.z, a01.w), make_float2(a23.x, a23.y),
                                   make_float2(a23.z, a23.w)};
              const float2 b[4] = {make_float2(b01.x, b01.y), make_float2(b01.z, b01.w), make_float2(b23.x, b23.y),
                                   make_float2(b23.z, b23.w)};
              // reO = Re(S_a S_b*) - Re(X_a X_b*), S = up + dn, X = ud + du
              // imO = Im(up_a up_b* + dn_a dn_b* - ud_a ud_b* - du_a du_b*)
              const float sax = a[0].x + a[1].x, say = a[0].y + a[1].y;
              const float sbx = b[0].x + b[1].x, sby = b[0].y + b[1].y;
              const float xax = a[2].x + a[3].x, xay = a[2].y + a[3].y;
              const float xbx = b[2].x + b[3].x, xby = b[2].y + b[3].y;
              reO = (sax * sbx + say * sby) - (xax * xbx + xay * xby);
              imO = (a[0].y * b[0].x - a[0].x * b[0].y) + (a[1].y * b[1].x - a[1].x * b[1].y) -
                    (a[2].y * b[2].x - a[2].x * b[2].y) - (a[3].y * b[3].x - a[3].x * b[3].y);
            }
          }
          p1[q] = w8[q] * reO;
          p2[q] = -w8[q] * imO;
        }
        uint4 h1, l1, h2, l2;
        split8(p1, h1, l1);
        split8(p2, h2, l2);
        const int o1 = core_off(pp, kg * 8, kM), o2 = core_off(kPairs + pp, kg * 8, kM);
        *reinterpret_cast<uint4*>(st + o1) = h1;
        *reinterpret_cast<uint4*>(st + kABytes + o1) = l1;
        *reinterpret_cast<uint4*>(st + o2) = h2;
        *reinterpret_cast<uint4*>(st + kABytes + o2) = l2;
      }
      async_proxy_fence();
      if (!(pl.fault == 1 && n == 0)) mbar_arrive(&afull[s]);
      // warps 0-3 (TMEM lanes 0-127) move the FP32 accumulator into the FP64
      // tile after the group's last chunk: 32 columns at a time through this
      // warp's 8 KB of the stage of chunk n (free until chunk n + 2, which
      // waits for these warps), then one bulk copy (first flush) or bulk
      // FP64 add into the tile. A flush starts once the previous one's bulk
      // operations completed, so the additions happen in a fixed order. Their
      // next A-full arrival tells the control warp that the accumulator and
      // the stage may be overwritten.
      if ((g == kFlushChunks - 1 || n == nch - 1) && wid < 4) {
        if (wait(&mdone[s], (n >> 1) & 1, 4)) {
          tc_fence_after();
          double* stg = reinterpret_cast<double*>(st) + wid * (32 * 32);
          double* dst = out + part_index(wid * 32, 0);
          if (lane == 0) bulk_wait_all();
          __syncwarp();
          for (int cb = 0; cb < kN; cb += 32) {
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(wid * 32) << 16) + cb;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            // the previous pass's bulk operation has read the staging block
            if (lane == 0) bulk_wait_read();
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 32; ++q) stg[q * 32 + lane] = (double)__uint_as_float(r[q]);
            async_proxy_fence();
            __syncwarp();
            if (lane == 0) bulk_store(dst + cb * 32, stg, 32 * 32 * sizeof(double), flushes > 0);
          }
          if (lane == 0) bulk_wait_read();
          __syncwarp();
          tc_fence_before();
        }
      }
      if (g == kFlushChunks - 1 || n == nch - 1) ++flushes;
    }
    // an empty range (or an abort before the first flush) still owns its
    // tile: the producers zero it
    if (flushes == 0)
      for (int idx = tid; idx < kM * kN; idx += kProducers) out[idx] = 0.0;
    // every bulk copy of this CTA has completed before it exits
    if (wid < 4 && lane == 0) bulk_wait_all();
  }
  __syncthreads();
  // drain: the last commit completes after every earlier MMA of the control
  // thread; it is waited for on every path before TMEM is freed
  const int nlast = *(volatile int*)s_last;
  if (tid == kProducers && nlast >= 0 && !mbar_wait(&mdone[nlast & 1], (nlast >> 1) & 1, pl.wait_ns))
    atomicExch(pl.err, 3);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (wid == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kN));
}

// Sums the FP64 partial tiles of each frequency tile's pieces in piece order
// and scatters rows to acc[2][9][np][nf] (P1 -> Im, P2 -> Re). 32 columns
// at a time go through shared memory so that both the reads of the tiles
// (part_index: rows fastest) and the writes of acc (frequency fastest)
// coalesce.
__global__ void __launch_bounds__(256) reduce_kernel(Plan pl, ContractArgs a) {
  constexpr int kCB = 32;
  __shared__ double sT[kM][kCB + 1];
  const int tile = blockIdx.x, ft = blockIdx.y;
  const int2 tb = pl.tiles[tile];
  const int2 ir = pl.ft_items[ft];
  const int A = 3 * a.neps;
  const size_t blk = (size_t)9 * a.np * a.nf;
  for (int cb = 0; cb < kN; cb += kCB) {
    for (int idx = threadIdx.x; idx < kM * kCB; idx += blockDim.x) {
      const int row = idx % kM, col = cb + idx / kM;
      double s = 0.0;
      for (int itm = ir.x; itm < ir.y; ++itm)
        s += pl.part[((size_t)itm * pl.ntile + tile) * (kM * kN) + part_index(row, col)];
      sT[row][col - cb] = s;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kM * kCB; idx += blockDim.x) {
      const int row = idx / kCB, c = idx % kCB;
      const int f = ft * kN + cb + c;
      if (f >= a.nf) continue;
      const int pp = row & (kPairs - 1);
      const int av = tb.x * 8 + (pp >> 3), bv = tb.y * 8 + (pp & 7);
      if (av >= A || bv >= A) continue;
      const int m = av / 3, i = av % 3, n = bv / 3, j = bv % 3;
      if (n > m) continue;
      const size_t o = ((size_t)(i * 3 + j) * a.np + (size_t)m * (m + 1) / 2 + n) * a.nf + f;
      if (row < kPairs)
        a.acc[blk + o] = sT[row][c];  // Im part
      else
        a.acc[o] = sT[row][c];  // Re part
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- host side
namespace {

struct HostPlan {
  std::vector<int> chunk_ft, chunk_t0, chunk_t1;
  std::vector<int4> items;
  std::vector<int2> ft_items, tiles;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

HostPlan make_plan(const ContractArgs& a, const int2* trange_host, int nft) {
  HostPlan h;
  const int A = 3 * a.neps, nb = (A + 7) / 8;
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      const int amax = std::min(8 * i + 7, A - 1), bmin = 8 * j;
      if (amax / 3 >= bmin / 3) h.tiles.push_back(make_int2(i, j));
    }
  long long total = 0;
  for (int ft = 0; ft < nft; ++ft) total += (trange_host[ft].y - trange_host[ft].x + kKC - 1) / kKC;
  // pieces: enough CTAs to fill the GPU a few times, each a multiple of the flush group
  const long long want = std::max<long long>(1, (kTargetCtas + (long long)h.tiles.size() - 1) / h.tiles.size());
  long long piece = std::max<long long>(kFlushChunks, (total + want - 1) / want);
  piece = (piece + kFlushChunks - 1) / kFlushChunks * kFlushChunks;
  h.ft_items.resize(nft);
  for (int ft = 0; ft < nft; ++ft) {
    const int tb = trange_host[ft].x, te = trange_host[ft].y;
    const int c0 = (int)h.chunk_ft.size();
    for (int t = tb; t < te; t += kKC) {
      h.chunk_ft.push_back(ft);
      h.chunk_t0.push_back(t);
      h.chunk_t1.push_back(te);
    }
    const int c1 = (int)h.chunk_ft.size();
    const int i0 = (int)h.items.size();
    for (int c = c0; c < c1; c += (int)piece) h.items.push_back(make_int4(ft, c, (int)std::min<long long>(c1, c + piece), 0));
    h.ft_items[ft] = make_int2(i0, (int)h.items.size());
  }
  return h;
}

}  // namespace

size_t mixed_workspace_bytes(const ContractArgs& a, long long T) {
  // upper bound: every transition in at most ceil((2W+N)/N)+1 frequency tiles
  const int nft = (a.nf + kN - 1) / kN;
  const long long span = a.window < 0 ? nft : std::min<long long>(nft, (2LL * a.window + kN) / kN + 2);
  const long long nchunk = (T * span + kKC - 1) / kKC + nft + 1;
  const int A = 3 * a.neps, nb = (A + 7) / 8;
  const long long ntile = (long long)nb * nb;
  const long long nitem = kTargetCtas + 2 * nft + 1;  // pieces: want + one remainder per frequency tile
  size_t b = 0;
  b += align256(sizeof(int) * 3 * nchunk);
  b += align256(sizeof(int4) * nitem);
  b += align256(sizeof(int2) * nft);
  b += align256(sizeof(int2) * ntile);
  b += align256(sizeof(float) * (T + 1));
  b += align256((size_t)kWChunkBytes * nchunk);
  b += align256(sizeof(double) * (size_t)nitem * ntile * kM * kN);
  b += align256(sizeof(int) * 4);
  b += align256(sizeof(float2) * (size_t)(T + 1) * A * a.nch);
  return b;
}

size_t mixed_smem_bytes(int nch) {
  const int nbuf = nch == 1 ? 2 : 1;  // overlap buffers of padded rows (see mixed_kernel)
  return (size_t)2 * (2 * kABytes + kWChunkBytes) + (size_t)nbuf * 16 * (kKC * nch + 2) * sizeof(float2) +
         (size_t)nbuf * kKC * sizeof(float) + 6 * sizeof(uint64_t) + 4 * sizeof(int);
}

// Precision diagnostic of the FP32 overlap copies: max ||M32|^2 - |M|^2| and
// max |M|^2 over all entries (non-negative doubles compare as integers).
__global__ void m32_error_kernel(const double2* __restrict__ M, const float2* __restrict__ M32, size_t n,
                                 unsigned long long* out) {
  double e = 0.0, mx = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = M[i];
    const float2 w = M32[i];
    const double a = v.x * v.x + v.y * v.y;
    const double b = (double)w.x * w.x + (double)w.y * w.y;
    e = fmax(e, fabs(a - b));
    mx = fmax(mx, a);
  }
  for (int o = 16; o > 0; o >>= 1) {
    e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(e));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(mx));
  }
}

__global__ void m_to_f32_kernel(const double2* __restrict__ M, float2* __restrict__ M32, size_t n,
                                const double* __restrict__ w, float* __restrict__ w32, long long T) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (M) {
      const double2 v = M[i];
      M32[i] = make_float2((float)v.x, (float)v.y);
    }
    if (i < (size_t)T) w32[i] = (float)w[i];
  }
}

cudaError_t launch_contract_mixed(const ContractArgs& a, long long T, void* ws, int& nlaunch, cudaStream_t st,
                                  long long* mmas) {
  nlaunch = 0;
  if (mmas) *mmas = 0;
  const int nft = (a.nf + kN - 1) / kN;
  // transition range of every 256-wide frequency tile (the FP64 tiles are 64 wide)
  std::vector<int2> tr(nft);
  {
    const int ft64 = contract_ftile();
    const int n64 = (a.nf + ft64 - 1) / ft64;
    std::vector<int2> t64(n64);
    cudaError_t e = cudaMemcpyAsync(t64.data(), a.trange, sizeof(int2) * n64, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    for (int ft = 0; ft < nft; ++ft) {
      int lo = INT32_MAX, hi = 0;
      for (int q = ft * (kN / ft64); q < std::min(n64, (ft + 1) * (kN / ft64)); ++q) {
        lo = std::min(lo, t64[q].x);
        hi = std::max(hi, t64[q].y);
      }
      if (lo > hi) lo = hi;
      tr[ft] = make_int2(lo, hi);
    }
  }
  HostPlan h = make_plan(a, tr.data(), nft);
  Plan pl{};
  pl.nft = nft;
  pl.ntile = (int)h.tiles.size();
  pl.nchunk = (int)h.chunk_ft.size();
  pl.nitem = (int)h.items.size();
  const int A = 3 * a.neps;
  uint8_t* p = reinterpret_cast<uint8_t*>(ws);
  auto take = [&](size_t bytes) {
    uint8_t* r = p;
    p += align256(bytes);
    return r;
  };
  pl.chunk_ft = reinterpret_cast<int*>(take(sizeof(int) * std::max(1, pl.nchunk)));
  pl.chunk_t0 = reinterpret_cast<int*>(take(sizeof(int) * std::max(1, pl.nchunk)));
  pl.chunk_t1 = reinterpret_cast<int*>(take(sizeof(int) * std::max(1, pl.nchunk)));
  pl.item = reinterpret_cast<int4*>(take(sizeof(int4) * std::max(1, pl.nitem)));
  pl.ft_items = reinterpret_cast<int2*>(take(sizeof(int2) * nft));
  pl.tiles = reinterpret_cast<int2*>(take(sizeof(int2) * std::max(1, pl.ntile)));
  pl.wgt32 = reinterpret_cast<float*>(take(sizeof(float) * (T + 1)));
  pl.wbuf = take((size_t)kWChunkBytes * std::max(1, pl.nchunk));
  pl.part = reinterpret_cast<double*>(take(sizeof(double) * (size_t)std::max(1, pl.nitem) * pl.ntile * kM * kN));
  pl.err = reinterpret_cast<int*>(take(sizeof(int) * 4));
  pl.wait_ns = a.wait_ns > 0 ? (uint64_t)a.wait_ns : kWaitNs;
  pl.fault = a.fault;
  float2* M32 = a.M32 ? const_cast<float2*>(a.M32)
                      : reinterpret_cast<float2*>(take(sizeof(float2) * (size_t)(T + 1) * A * a.nch));
  if ((size_t)(p - reinterpret_cast<uint8_t*>(ws)) > mixed_workspace_bytes(a, T)) return cudaErrorInvalidValue;
  cudaError_t e;
#define PMX_CP(dst, src, n)                                                                            \
  if ((n) > 0) {                                                                                      \
    e = cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st);                                     \
    if (e != cudaSuccess) return e;                                                                   \
  }
  PMX_CP(pl.chunk_ft, h.chunk_ft.data(), sizeof(int) * pl.nchunk);
  PMX_CP(pl.chunk_t0, h.chunk_t0.data(), sizeof(int) * pl.nchunk);
  PMX_CP(pl.chunk_t1, h.chunk_t1.data(), sizeof(int) * pl.nchunk);
  PMX_CP(pl.item, h.items.data(), sizeof(int4) * pl.nitem);
  PMX_CP(pl.ft_items, h.ft_items.data(), sizeof(int2) * nft);
  PMX_CP(pl.tiles, h.tiles.data(), sizeof(int2) * pl.ntile);
#undef PMX_CP
  e = cudaMemsetAsync(pl.err, 0, sizeof(int) * 4, st);
  if (e != cudaSuccess) return e;
  // zero the accumulators: tiles with no transitions are written by reduce_kernel only where pieces exist
  e = cudaMemsetAsync(a.acc, 0, sizeof(double) * 2 * 9 * (size_t)a.np * a.nf, st);
  if (e != cudaSuccess) return e;
  if (T > 0) {
    // FP32 copies of the overlaps (unless they come in FP32) and of the weights
    m_to_f32_kernel<<<1184, 256, 0, st>>>(a.M32 ? nullptr : a.M, M32, a.M32 ? (size_t)T : (size_t)T * A * a.nch,
                                          a.wgt, pl.wgt32, T);
    ++nlaunch;
    if (a.stats && a.M) {
      e = cudaMemsetAsync(a.stats, 0, 2 * sizeof(double), st);
      if (e != cudaSuccess) return e;
      m32_error_kernel<<<592, 256, 0, st>>>(a.M, M32, (size_t)T * A * a.nch,
                                              reinterpret_cast<unsigned long long*>(a.stats));
      ++nlaunch;
    }
  }
  if (pl.nchunk > 0) {
    wgen_kernel<<<pl.nchunk, 256, 0, st>>>(pl, a);
    ++nlaunch;
  }
  if (pl.nitem > 0 && pl.ntile > 0) {
    const size_t sm = mixed_smem_bytes(a.nch);
    dim3 grid(pl.ntile, pl.nitem);
    if (a.nch == 1) {
      e = cudaFuncSetAttribute(mixed_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      if (e != cudaSuccess) return e;
      mixed_kernel<1><<<grid, kThreads, sm, st>>>(pl, a, M32);
    } else {
      e = cudaFuncSetAttribute(mixed_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      if (e != cudaSuccess) return e;
      mixed_kernel<4><<<grid, kThreads, sm, st>>>(pl, a, M32);
    }
    ++nlaunch;
    reduce_kernel<<<dim3(pl.ntile, nft), 256, 0, st>>>(pl, a);
    ++nlaunch;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int err = 0;
  e = cudaMemcpyAsync(&err, pl.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  if (err != 0) return cudaErrorTimeout;
  // every chunk is multiplied by every pair tile: 3 products x 2 K steps
  if (mmas) *mmas = 6LL * pl.ntile * pl.nchunk;
  return cudaSuccess;
}

}  // namespace dev
}  // namespace pmx
