// Argument blocks and launchers of the chi-stage kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pmx {
namespace dev {

struct OverlapArgs {
  int n;            // eigenvector length (npw, or 2 npw with SOC)
  int npw;
  int soc;          // eigenvectors are spinors
  int nev;          // eigenvectors stored per k
  int neps;
  int nch;          // 1 or 4 output channels
  int mode;         // 0 epsij, 1 epsLL
  int cchunk;       // conduction states per CTA
  int vchunk;       // valence states per CTA
  int ncd_max, nvd_max;
  const double2* zk;      // [nk][nev][n] eigenvectors at k
  const double2* zq;      // [nk][nev][n] eigenvectors at k+q
  const int* ncd;         // [nk] distinct conduction states
  const int* nvd;         // [nk] distinct valence states
  const int* cbase;       // [nk] offset into cidx
  const int* vbase;       // [nk] offset into vidx
  const int* cidx;        // eigenvector index of each conduction state
  const int* vidx;        // eigenvector index of each valence state
  const long long* blkoff;  // [nk] offset of the k block in dest
  const long long* dest;    // sorted transition of (k, c, v), -1 if unused
  const int* loci;        // [neps][npw]
  const double* G;        // [npw][3]
  const double* kpts;     // [nk][3]
  double q[3];
  const double2* uvec;    // [neps][3][3]  u_i of q + G_m
  const double2* ssoc;    // [neps][3]     u_i^H v_soc(G_m)
  double2* M;             // [T][3 neps][nch]
};

// Device transition list of one q (trans.cu).
constexpr int kTransMaxNB = 512;  // NBAND limit (per-thread state lists)
struct TransSummary {
  long long T;     // transitions
  long long nblk;  // (k, c, v) slots of dest
  int ncd_max, nvd_max;
  int cuts, ties;  // degenerate NBAND cuts, states within 1e-8 eV of E_ref
  int f0_lo, f0_hi;
};
struct TransArgs {
  const double* wk;  // [nk][nval] eigenvalues at k (spatial states without SOC)
  const double* wq;  // [nk][nval] at k+q
  const double* kw;  // [nk] k-point weights
  int nk, nval, nband, nh, soc, xyz;
  double off, w0, df;
  // per k
  int *ncd, *nvd, *cbase, *vbase, *cidx, *vidx, *ntr, *nblk;  // cidx/vidx [nk][nband]
  long long *blkoff, *toff;
  // transitions in k order
  long long* rsrc;
  double *rde, *rw;
  int* rf0;
  // sorted by window start
  long long* dest;  // [nblk] sorted index of (k, c, v), -1 if unused
  double *de, *wgt;
  int* f0;
  int2* trange;     // [nft] transition range of every frequency tile
  int *cnt, *btot;  // sort scratch (transitions_sort_ints)
  TransSummary* sum;
};
// occupations, counts and offsets; the summary (device) is complete when the
// stream reaches it
cudaError_t launch_transitions_count(const TransArgs& a, cudaStream_t st);
// the list, sorted by window start when asked, and the frequency-tile ranges
// (window < 0: every tile takes all transitions)
cudaError_t launch_transitions_fill(const TransArgs& a, const TransSummary& s, bool sort, int nft, int ftile, int nf,
                                    int window, cudaStream_t st);
size_t transitions_sort_ints(const TransSummary& s);
bool transitions_sortable(const TransSummary& s);

// Overlaps of the mixed path on the tensor cores (overlap_tc.cu): the same
// moments as overlap_kernel from split TF32 operands, FP32 results M32[t][3 neps][nch].
constexpr int kOvlTcMaxN = 128;  // GEMM columns (c, s, w) per CTA
struct OverlapTcArgs {
  OverlapArgs a;      // M unused
  float2* M32;
  long long wait_ns;  // limit of the bounded mbarrier waits (0: 2 s)
  int* err;           // set to 1 when a wait ran out
  int fault;          // tests only: 4 = the first chunk's MMAs are not committed, so that a wait runs out
};
cudaError_t launch_overlap_tc(const OverlapTcArgs& t, int nk, cudaStream_t st);
size_t overlap_tc_smem_bytes(int npw, int neps);

struct ContractArgs {
  const double2* M;     // [T][3 neps][nch] (may be null on the mixed path when M32 is given)
  const float2* M32;    // mixed path: overlaps already in FP32 (tensor-core overlaps), or null
  const double* dE;     // [T]
  const double* wgt;    // [T] k weight times spin multiplicity
  const int* f0;        // [T] window centre int((dE - w0)/dw)
  const int2* trange;   // [n f-tiles] transition range of each frequency tile
  int neps, np, nf, nch;
  int window;           // half width, or -1 for all frequencies
  int delta;            // broadening model
  double eps, dfreq;
  double* acc;          // [2][9][np][nf] Re then Im
  double* acc_pv;       // principal-value accumulators (epsLL, kk = 0) or null
  double* stats;        // mixed path only, optional (device, 2 doubles): max ||M32|^2 - |M|^2|, max |M|^2
                       // (needs M)
  int pvclass;          // principal-value function: 0 by (i, j) block (epsLL), 3 = 1/dE/(dE^2-w^2) for all (epsxyz)
  long long wait_ns;    // mixed path: limit of every bounded mbarrier wait (0: 2 s)
  int fault;            // mixed path, tests only: 1 = the producers withhold their first A-full arrival,
                        // so that the control thread's wait runs out (the timeout path is exercised)
};

struct ScaleArgs {
  int mode;             // 0 epsij, 1 epsLL, 2 epsxyz
  int np, nf;
  double dfreq;
  double sf;            // epsij SCALEFACTOR
  double sf_ll, sf_lt, sf_tt;
  const double* qgn;    // [neps] |q + G_m|
  const double* acc;
  const double* acc_pv;
  double* out;
};

cudaError_t launch_overlap(const OverlapArgs& a, int nk, cudaStream_t st);
size_t overlap_smem_bytes(int cchunk, int vchunk, int n, int npw);
// Largest conduction / valence chunks whose staged eigenvectors fit 200 KB of
// shared memory; false when even one of each does not fit.
bool overlap_tiles(int ncd_max, int nvd_max, int n, int npw, int& cchunk, int& vchunk);
// Tile shapes the autotuner may try for overlap_kernel (at most maxc): first
// the largest chunks (overlap_tiles), then those with the conduction and/or
// valence chunk halved (more CTAs per k-point, fewer eigenvectors staged per
// CTA, more CTAs per SM). Every shape computes the same M. Returns the count
// (0: no shape fits).
int overlap_tile_candidates(int ncd_max, int nvd_max, int n, int npw, int* cc, int* vc, int maxc);
cudaError_t launch_contract_f64(const ContractArgs& a, cudaStream_t st);
int contract_ftile();
cudaError_t launch_scale(const ScaleArgs& s, cudaStream_t st);
cudaError_t launch_kk(const double* chi, double* out, int rows, int nf, double dfreq, cudaStream_t st);

}  // namespace dev
}  // namespace pmx

namespace pmx {
namespace dev {
// eps_M per (q, w) from the chi LL block laid out [q][pair][f] (re, im);
// out [nq][nf] complex. neps <= 64.
cudaError_t launch_epsm(const double* re, const double* im, int neps, int nq, int nf, double2* out, cudaStream_t st);
// loss [nq][nf] = -Im(1/eps_M); peak [nq][2] = (frequency, height) of the
// largest loss at f >= fmin, refined by a parabola through its neighbours.
cudaError_t launch_loss(const double2* epsm, int nq, int nf, int fmin, double dfreq, double* loss, double* peak,
                        cudaStream_t st);
}  // namespace dev
}  // namespace pmx
