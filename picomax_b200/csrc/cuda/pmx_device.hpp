// Device-side data structures and kernel launchers of the picomax B200 path.
//
// Stage 1 (EPM): every (crystal, k) work item builds H(k) in HBM and is
// diagonalised by one CTA of the batched FP64 eigensolver. Stage 2 (chi):
// overlaps, transition list, the delta-weighted contraction and the
// Kramers-Kronig transform. Everything is stream-ordered on the caller's
// stream; nothing here allocates.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pmx {
namespace dev {

// One crystal as the kernels see it. Tables are indexed by an hkl difference
// d = (dh, dk, dl) through ((dh+2imax)*side + dk+2imax)*side + dl+2imax.
struct CrystalDev {
  int npw;        // plane waves N_G
  int soc;        // 1: spinor H of size 2 N_G; 0: H0 of size N_G (spectrum doubled)
  int imax;       // |h|,|k|,|l| <= imax for every G
  int side;       // 4*imax+1
  double kin;     // KCON (2 pi / a)^2, eV
  const double* G;      // [npw][3], units 2 pi / a
  const int* hkl;       // [npw][3]
  const double2* vloc;  // V(G_i - G_j) in eV for d = hkl_i - hkl_j (0 beyond g2max)
  const double2* vso;   // VSO(q) = lambda_S cos_sum + i lambda_A sin_sum, eV, d = hkl_j - hkl_i
};

// One eigenproblem of the batch.
struct EigItem {
  int crystal;        // index into the crystal table
  int n;              // matrix dimension (npw, or 2 npw with SOC)
  int nev;            // lowest eigenvectors returned (when want_vec)
  int nval;           // lowest eigenvalues returned, nval >= nev
  int want_vec;       // 1: also eigenvectors
  double k[3];        // wave vector, units 2 pi / a
  long long h_off;    // double2 offset of the n*n column-major workspace
  long long w_off;    // double offset of nval eigenvalues
  long long z_off;    // double2 offset of nev eigenvectors (column s at z_off + s*n)
  long long s_off;    // double offset of the item's scratch (heev_scratch_doubles)
  int ld;             // leading dimension of the matrix (0: n); rows n..ld-1 and columns
                      // n..ld-1 of the workspace are zero when ld > n
  long long r_off;    // double2 offset of the two-stage path's band reflectors (heev2_rbuf_double2)
  int bisect_cap;     // rounds of the eigenvalue bisection at most (0: the default cap; tests set 1)
  long long wait_ns;  // limit of one bounded wait of the two-stage bulge chase (0: 2 s)
  int wait_fault;     // tests only: 1 makes the bulge chase's sweep 1 wait for progress never made
};

// Fills H(k) of every item (full Hermitian storage, leading dimension
// EigItem::ld, padding rows and columns zero) into hbuf.
cudaError_t launch_assemble(const CrystalDev* crystals, const EigItem* items, int nitems,
                            int max_npw, double2* hbuf, cudaStream_t st);

// Eigensolve of every item. Matrices with n <= smem_max_n run with the matrix
// resident in shared memory. info[i] != 0 flags a failure of item i.
// variant selects the global-memory path schedule (see heev_variants); the
// resident path ignores it.
// tri (optional, [nitems][4 n]): per item d[n], e[n] (e[n-1] = 0) and the
// reflector scalars tau[n] (complex) of H = Q T Q^H; with it, the reflectors
// are left in hbuf (column j, rows > j, v[j+1] = 1) on every path.
cudaError_t launch_heev(const EigItem* items, int nitems, int max_n, int max_nev, double2* hbuf,
                        double* wbuf, double2* zbuf, double* scratch, int* info, cudaStream_t st, int variant = 0,
                        double* tri = nullptr);
int heev_smem_max_n();
// Global scratch (doubles) one item of size n with nvec eigenvectors needs in
// a launch whose largest matrix is max_n; items must be spaced by at least
// this much (EigItem::s_off), and the scratch is used with or without vectors
// when max_n > 832.
size_t heev_scratch_doubles(int n, int nvec, int max_n);
// Number of schedules launch_heev offers for matrices of size max_n.
int heev_variants(int max_n, int max_nev);
// Batch size unit of the eigensolver on the current device: the SM count
// times the least common multiple of the resident CTAs per SM of every
// schedule for (max_n, max_nev). A batch that is a multiple of it fills every
// wave of CTAs whichever schedule runs.
int heev_batch_unit(int max_n, int max_nev);

// Two-stage eigensolver (eig2.cu): dense -> band (16 sub-diagonals) on the
// FP64 tensor cores, band -> tridiagonal by bulge chasing (the band in
// shared memory up to ld = 416, in rbuf up to 832), bisection + inverse
// iteration, back-transforms. Items carry ld = heev2_ld(n) (the workspace
// padded with zeros, see launch_assemble) and r_off, spaced by at least
// heev2_rbuf_double2(ld, heev2_ld(max_n)) double2 in rbuf (max_n: the
// launch's largest n).
int heev2_ld(int n);
bool heev2_supported(int max_n);
size_t heev2_rbuf_double2(int ld, int launch_ld);
cudaError_t launch_heev2(const EigItem* items, int nitems, int max_n, int max_nval, int max_nvec, double2* hbuf,
                         double* wbuf, double2* zbuf, double* scratch, double2* rbuf, int* info, cudaStream_t st);

// Symmetry reduction of a Gamma-centred n[0] x n[1] x n[2] grid (kgrid.cu):
// ops are integer matrices in the reciprocal basis (a group, identity
// included) that map the grid onto itself. rep/cnt: device scratch of
// n0 n1 n2 ints each; idx [nirr][3] (may be null) and w [nirr] receive the
// representatives (smallest linear index of each orbit, index order) and
// their orbit sizes; nirr (device) their count.
constexpr int kKgridMaxOps = 96;
struct KgridOps {
  int n;
  int m[kKgridMaxOps][9];
};
cudaError_t launch_kgrid_reduce(const KgridOps& ops, const int* n, int* rep, int* cnt, int* idx, int* w, int* nirr,
                                cudaStream_t st);

}  // namespace dev
}  // namespace pmx
