// Reverse-mode (adjoint) kernels of the band and chi_LL -> eps_M stages.
//
// The loss gradient flows eps_M -> chi_LL (matrix inverse) -> Kramers-Kronig
// (transpose) -> scale -> contraction over transitions (per-transition
// overlap and energy adjoints) -> overlaps (eigenvector adjoints) -> the
// Hermitian eigenproblem (Hellmann-Feynman plus the eigenvector term, with
// degenerate pairs masked) -> H(k) -> form factors and SOC parameters.
// Everything is FP64.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace pmx {
namespace dev {

// eps_M adjoint per (q, w): from the chi LL block [q][pair][f] (re, im) and
// the upstream gradient g [q][f] = (dL/dRe eps_M, dL/dIm eps_M), writes
// dL/dRe chi, dL/dIm chi of every stored pair [q][pair][f]. neps <= 64.
cudaError_t launch_epsm_vjp(const double* re, const double* im, const double2* g, int neps, int nq, int nf,
                            double* gre, double* gim, cudaStream_t st);

// Transposed Kramers-Kronig on [2][rows][nf] (Re block then Im block):
// out_Re = g_Re + ds K^T g_Im, out_Im = g_Im + ds K^T g_Re.
cudaError_t launch_kk_t(const double* g, double* out, int rows, int nf, double dfreq, cudaStream_t st);

struct ContractVjpArgs {
  const double2* M;     // [T][3 neps][1]: L overlap of pair m at row 3 m
  const double* dE;     // [T]
  const double* wgt;    // [T]
  int T, neps, np, nf;
  int delta;            // broadening model
  double eps, dfreq;
  const double* gre;    // [np][nf] dL/dRe chi_LL (after the KK transpose)
  const double* gim;    // [np][nf] dL/dIm chi_LL
  const double* f1;     // [np] pi * SF_LL / (|q+G_m| |q+G_n|) (applies for f >= 1)
  const double* f2;     // [np] 2 SF_LL / (|q+G_m| |q+G_n|) principal-value factor, or null (kk on)
  double2* obar;        // [T][np] dL/dO of O_mn = M_m conj(M_n)
  double* dEbar;        // [T] dL/d(E_c - E_v), accumulated (zero it first)
};
cudaError_t launch_contract_vjp(const ContractVjpArgs& a, cudaStream_t st);

// dL/dM_m = sum_n obar_mn M_n + sum_n conj(obar_nm) M_n  -> mbar [T][neps]
cudaError_t launch_mbar(const double2* M, const double2* obar, int T, int neps, double2* mbar, cudaStream_t st);

struct ZbarArgs {
  int nk;               // k-points of the block
  int n, npw, soc;
  int nev;              // eigenvectors stored per k (zk/zq stride)
  int ns;               // columns of zbar/lbar per k
  int neps;
  int ncd_max, nvd_max;
  const double2* zk;    // [nk][nev][n] at k (conduction)
  const double2* zq;    // [nk][nev][n] at k+q (valence)
  const int *ncd, *nvd, *cbase, *vbase, *cidx, *vidx;
  const long long *blkoff, *dest;
  const int* loci;      // [neps][npw]
  const int* linv;      // [neps][npw]: p with loci[m][p] = r, or -1
  const double2* mbar;  // [T][neps]
  const double* dEbar;  // [T]
  double2* zbar_k;      // [nk][ns][n] (written for the states in use, others untouched)
  double2* zbar_q;
  double* lbar_k;       // [nk][ns]
  double* lbar_q;
};
cudaError_t launch_zbar(const ZbarArgs& a, cudaStream_t st);

// Batched complex GEMM, column-major: C_b = op(A_b) B_b with op = identity
// (conj_a = 0) or conjugate transpose (conj_a = 1). A_b is (conj_a ? K x M :
// M x K) with leading dimension lda and batch stride sa; B_b is K x N (ldb,
// sb); C_b is M x N (ldc, sc).
cudaError_t launch_zgemm_batched(int conj_a, int M, int N, int K, const double2* A, int lda, long long sa,
                                 const double2* B, int ldb, long long sb, double2* C, int ldc, long long sc,
                                 int batch, cudaStream_t st);

// Eigenvector-adjoint kernel matrix, in place on C = Z^H Zbar ([batch][ns][nall],
// column j of item b at C + (b ns + j) nall): K_mj = (C_mj - conj(C_jm)) /
// (2 (lam_j - lam_m)) for m < ns, C_mj / (lam_j - lam_m) for m >= ns, zero
// where |lam_j - lam_m| < tau, and K_jj = lbar_j.
cudaError_t launch_eig_kmat(double2* C, const double* lam, int lam_stride, const double* lbar, int nall, int ns,
                            int batch, double tau, cudaStream_t st);

struct ResolventArgs {
  int n;                // matrix dimension (<= 1216)
  int ns;               // right-hand sides per item (states with a gradient)
  int nsx;              // eigenvectors projected out (a prefix of the spectrum, nsx >= ns)
  int nitems;
  const double2* H;     // [item][n][n] reflectors left by launch_heev(tri)
  const double* tri;    // [item][4 n] d, e, tau of launch_heev(tri)
  const double* lam;    // eigenvalues, item b at lam + b lam_stride
  int lam_stride;
  const double2* Z;     // eigenvectors, item b at Z + b zs, column m at m n (m < nsx)
  long long zs;
  const double2* zbar;  // [item][ns][n]
  double2* Y;           // [item][ns][n], accumulated: Y += P (lam_k - H)^-1 P zbar_k
  double* work;         // [item][8][5 n] doubles
};
cudaError_t launch_resolvent(const ResolventArgs& a, cudaStream_t st);

// X = diag(lbar) Z (Hellmann-Feynman only): X [batch][ns][n], Z stride zs.
cudaError_t launch_hf_x(const double2* Z, long long zs, const double* lbar, int n, int ns, int batch, double2* X,
                        cudaStream_t st);

// Pair accumulators R over items: R[w][s][i][j] += sum_b wt_w(k_b) sum_j'
// conj(X_b[(i s1), j']) Z_b[(j s2), j'], s = 2 s1 + s2, w: weights 1, kx,
// ky, kz (spinor) or R[i][j] (no SOC, weight 1). X [batch][ns][n] (stride xs),
// Z [batch][..][n] (stride zs), kpts [batch][3].
cudaError_t launch_hgrad(const double2* X, long long xs, const double2* Z, long long zs, const double* kpts,
                         int batch, int n, int npw, int soc, int ns, double2* R, cudaStream_t st);

// Scatter R onto the hkl-difference tables of the form factors:
// SV[d] += sum_s R[0][ss](i, j), d = hkl_i - hkl_j; SSO[d'] += i sum_x s_x T^x
// with s = (k + G_j) x (k + G_i), d' = hkl_j - hkl_i.
cudaError_t launch_hscatter(const double2* R, int npw, int soc, const int* hkl, const double* G, int imax,
                            double2* SV, double2* SSO, cudaStream_t st);

}  // namespace dev
}  // namespace pmx
