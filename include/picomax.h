/*
 * picomax.h - C-ABI of the B200 implementation of PicoMax's two hot stages:
 * the EPM band solve and the chi(q, w) local-field accumulation.
 *
 * The reference exposes no library API: its only interface is the `picomax`
 * executable (argv in, binary .dat/.gpt files out). These entry points are
 * the functions that executable is built from, one per reference stage, with
 * plain pointers and sizes. A status code replaces the reference's abort().
 *
 * Host buffers are caller-owned. Device work is ordered on the context's
 * stream; every call below returns after its results are in the caller's
 * buffers unless the name ends in _async.
 */
#ifndef PICOMAX_B200_H_
#define PICOMAX_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  PMX_OK = 0,
  PMX_ERR_INVALID = 1,     /* bad argument or option (reference: abort()) */
  PMX_ERR_CUDA = 2,        /* CUDA runtime error */
  PMX_ERR_NOCONV = 3,      /* eigensolver did not converge (reference: abort() at src/pmx_epm.cpp:233) */
  PMX_ERR_TIMEOUT = 4,     /* a bounded device wait ran out */
  PMX_ERR_NO_DEVICE = 5,   /* no CUDA device: this library has no CPU path */
  PMX_ERR_UNSUPPORTED = 6, /* input outside what this library implements */
  PMX_ERR_LIMIT = 7,       /* size beyond the fixed maximum of pmx_heev_batched_noalloc, or of pmx_write_npz */
  PMX_ERR_IO = 8           /* a file could not be written */
} pmx_status;

typedef enum {
  PMX_SWITCH_NONE = 0,
  PMX_SWITCH_BAND = 1,
  PMX_SWITCH_EPSIJ = 2,
  PMX_SWITCH_EPSLL = 3,
  PMX_SWITCH_EPSXYZ = 4
} pmx_switch;
typedef enum { PMX_PREC_FP64 = 0, PMX_PREC_MIXED = 1 } pmx_precision;

typedef struct pmx_problem pmx_problem; /* parsed picomax invocation (host) */
typedef struct pmx_ctx pmx_ctx;         /* device context: stream, workspaces */

typedef struct {
  int npw;        /* plane waves N_G (NPW) */
  int nh;         /* reference Hamiltonian dimension 2 N_G */
  int soc;        /* 1 when any spin-orbit form factor is non-zero */
  int neps;       /* local-field G count (NEPS) */
  int nband;      /* NBAND */
  int nvalence;   /* -nvalence */
  int nk;         /* k-points (NKPT) */
  int nq;         /* q-points (NQ) */
  int nfreq;      /* NFREQ */
  int natom;      /* NATOM */
  int sw;         /* pmx_switch from -switch */
  int debug;      /* -debug level */
  int kk;         /* -kk */
  int delta;      /* -delta */
  double epsilon; /* -epsilon, eV */
  double dfreq;   /* -dfreq, eV */
  double a;       /* lattice constant, Angstrom */
  double gcut;    /* cutoff in 2 pi / a */
  double bz_volume;
  long long chi_values; /* doubles in one of the Re/Im blocks of the chi .dat */
} pmx_problem_info;

/* ---------------------------------------------------------------- problem */

/* Parses argv exactly as the reference does and builds the G list, loci table
 * and k/q lists. Replaces inputParser + inputProcess + init_crystal +
 * init_mater + generate_gpt/_rect + generate_loci + import_kpt/generate_kpt_*
 * (src/pmx.hpp:190-245, src/pmx_io.cpp:108-503, src/pmx_basis.cpp:29-355,
 * called from src/pmx.cpp:64-156). argv[0] is the program name. */
int pmx_problem_create(int argc, const char* const* argv, pmx_problem** out);
void pmx_problem_destroy(pmx_problem* p);
int pmx_problem_get_info(const pmx_problem* p, pmx_problem_info* info);
/* G vectors [npw][3] (units 2 pi / a) and their integer coordinates [npw][3];
 * the order is the reference's (src/pmx_basis.cpp:54-80). Either may be NULL. */
int pmx_problem_gvectors(const pmx_problem* p, double* G, int* hkl);
/* loci[m][p] = index of G_p + G_m or -1, [neps][npw] (src/pmx_basis.cpp:142-179). */
int pmx_problem_loci(const pmx_problem* p, int* loci);
/* k-points [nk][3] and weights [nk] (src/pmx_basis.cpp:200-650). */
int pmx_problem_kpoints(const pmx_problem* p, double* K, double* KW);
/* q-points [nq][3] (src/pmx_io.cpp:255-309). */
int pmx_problem_qpoints(const pmx_problem* p, double* Q);
/* Writes the text of `-debug 2/3` (printInput, src/pmx_io.cpp:510-614) to buf
 * (NUL-terminated, truncated at len). Returns the full length in *needed. */
int pmx_problem_dump(const pmx_problem* p, char* buf, size_t len, size_t* needed);
/* Writes ${wdir}/${out}.gpt (export_gpt, src/pmx_io.cpp:816-826). */
int pmx_problem_write_gpt(const pmx_problem* p);
/* Reusable output in place of the reference's planned HDF5 export
 * (src/pmx_io.cpp:744-807, commented out there; no HDF5 library here): count
 * float64 arrays in C order written to path as an uncompressed NumPy .npz
 * (a ZIP archive of NPY 1.0 files, readable by numpy.load). names[i] is the
 * array name (".npy" is appended), ndims[i] its rank, shapes the ranks'
 * extents one array after another. Files beyond 4 GB (no ZIP64) return
 * PMX_ERR_LIMIT, a failed write PMX_ERR_IO. The CLI writes ${out}.npz with
 * `-npz 1` (band: eband [nq][nband], qpoints [nq][3]; chi: ReXij and ImXij in
 * the .dat layout [3][3][nq][neps (neps + 1) / 2][nfreq], pairs [...][2] =
 * (m, n <= m) of the packed index, freq [nfreq] eV, qvec [nq][3], gvec
 * [neps][3] in 2 pi / a). No reference counterpart in working code. */
int pmx_write_npz(const char* path, int count, const char* const* names, const double* const* data, const int* ndims,
                  const long long* shapes);

/* ---------------------------------------------------------------- context */

/* Limit in nanoseconds of every bounded device wait (0: 2 s): the mbarrier
 * waits of the mixed-precision contraction and the waits of the two-stage
 * eigensolver's bulge chase on the previous sweep. A contraction wait that
 * runs out makes its CTA record the error, wait for its own copies and MMAs
 * in flight, free its tensor memory and return; a bulge-chase wait that runs
 * out fails its matrix. The call then fails with PMX_ERR_TIMEOUT and the
 * context stays usable. No reference counterpart (the reference has no device
 * waits). */
int pmx_ctx_set_wait_limit(pmx_ctx* ctx, long long ns);

/* Overlaps of the mixed-precision path (no reference counterpart): 3 on the
 * tensor cores from split TF32 operands (tcgen05 kind::tf32, FP32
 * accumulation); 0 in FP64 on the CUDA cores, rounded to FP32; 1 (default)
 * the faster of the two for the problem: the tensor cores without spin-orbit
 * coupling, FP64 with it; 2 both, the tensor-core results used and their
 * error against the FP64 ones reported by pmx_ctx_overlap_error. The FP64
 * path always uses FP64 overlaps. */
int pmx_ctx_set_overlap_mode(pmx_ctx* ctx, int mode);

/* Test hooks, no reference counterpart: fault 1 makes the producer warps of
 * the mixed contraction withhold their first A-full arrival, so that the
 * control warp's bounded wait runs out and the timeout path above runs
 * (combine with a short pmx_ctx_set_wait_limit); fault 2 stops the
 * eigensolver's bisection after one round, so that its status reports
 * non-convergence (PMX_ERR_NOCONV); fault 3 makes the second sweep of the
 * two-stage eigensolver's bulge chase wait for progress that never comes, so
 * that its bounded wait gives up (PMX_ERR_TIMEOUT; combine with a short
 * pmx_ctx_set_wait_limit); fault 4 leaves the first chunk of the tensor-core
 * overlaps uncommitted, so that the wait for its stage runs out
 * (PMX_ERR_TIMEOUT). 0 restores normal operation. */
int pmx_ctx_set_fault(pmx_ctx* ctx, int fault);

int pmx_ctx_create(int device, pmx_ctx** out);
void pmx_ctx_destroy(pmx_ctx* ctx);
/* Message of the last failing call on this context (NUL-terminated). */
const char* pmx_ctx_last_error(const pmx_ctx* ctx);
/* Device time of the stages of the last call, milliseconds:
 * [0] H assembly + eigensolves, [1] overlaps, [2] contraction, [3] scaling + KK,
 * [4] host<->device copies. Entries not run are 0. */
int pmx_ctx_stage_times(const pmx_ctx* ctx, double* ms5);
/* Launch count of this library's kernels since the context was created. */
long long pmx_ctx_kernel_launches(const pmx_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events after the library's. */
void* pmx_ctx_stream(const pmx_ctx* ctx);
/* Accumulated device time (CUDA events on the context stream around each
 * launch) and launch count of one kernel family since the context was
 * created: "assemble", "heev", "overlap", "contract_f64", "contract_mixed",
 * "scale", "kk". */
int pmx_ctx_kernel_time(const pmx_ctx* ctx, const char* family, double* ms, long long* launches);
/* Precision of the mixed path's FP32 overlap operands in the last pmx_chi*
 * call: max over all transitions and G of ||M_fp32|^2 - |M|^2| and max |M|^2.
 * New diagnostic (no reference counterpart). */
int pmx_ctx_overlap_error(const pmx_ctx* ctx, double* max_abs2_err, double* max_abs2);
/* Tensor-core work of the mixed path: tcgen05 MMA instructions (M 128, N 256,
 * K 16, BF16 operands, 2*128*256*16 flop each; the split products hi*hi,
 * hi*lo and lo*hi counted separately) issued by the mixed contractions of
 * this context so far. New diagnostic (no reference counterpart). */
int pmx_ctx_mixed_mmas(const pmx_ctx* ctx, long long* mmas);
/* Autotuner (on by default): the first batch of at least 148 matrices of a
 * given size times every eigensolver schedule once, and the first FP64
 * overlap launch over at least 148 k-points of a given shape times every tile
 * shape of pmx::dev::overlap_tile_candidates once (all give the same
 * overlaps); the fastest is kept for the rest of the context's life. No
 * reference counterpart. */
int pmx_ctx_set_autotune(pmx_ctx* ctx, int on);
/* Fixes the eigensolver schedule (0 = direct loads, then the prefetch and
 * shared-memory-partials schedules the matrix size allows; an index beyond
 * the last one means the last) for every later batch; -1 returns to the
 * autotuner. For tests that compare the schedules. No reference counterpart. */
int pmx_ctx_set_schedule(pmx_ctx* ctx, int schedule);
/* The autotuner's choices and trial times as JSON text (NUL-terminated,
 * truncated at len; full length in *needed). */
int pmx_ctx_tuning(const pmx_ctx* ctx, char* buf, size_t len, size_t* needed);
/* Bytes copied host->device and device->host by this context so far. */
int pmx_ctx_transfer_bytes(const pmx_ctx* ctx, long long* h2d_bytes, long long* d2h_bytes);
/* k and k+q points of the last pmx_chi* call at which the NBAND window cut a
 * degenerate set (|E_NBAND-1 - E_NBAND| < 1e-8 eV). There the reference's
 * result depends on its eigensolver's basis inside the set; a warning is
 * printed on stderr. No reference counterpart (new diagnostic). */
int pmx_ctx_degenerate_cuts(const pmx_ctx* ctx);
/* k and k+q points of the last pmx_chi* call with a state of the NBAND window
 * within 1e-8 eV of the reference energy (metals): the occupation test
 * E - E_ref > 0 of src/pmx_chi.cpp:391-397 is then decided by rounding, for the
 * reference as for this library; a warning is printed. No reference counterpart. */
int pmx_ctx_occupation_ties(const pmx_ctx* ctx);

/* ---------------------------------------------------------------- stage 1 */

/* Hamiltonian H(k) of every k in kpts [nk][3], full Hermitian storage,
 * column-major, complex interleaved: out [nk][nh][nh][2] with nh = 2 npw
 * (the spinor matrix of HamiltonianEPM, src/pmx_epm.cpp:56-153). */
int pmx_hamiltonian(pmx_ctx* ctx, const pmx_problem* p, const double* kpts, int nk, double* out);

/* Lowest nev eigenvalues (ascending) and optionally eigenvectors of a batch of
 * Hermitian matrices A [batch][n][n][2] (column-major, complex interleaved).
 * w [batch][nev]; z [batch][nev][n][2] or NULL. Replaces the
 * Eigen::SelfAdjointEigenSolver calls at src/pmx_epm.cpp:232 and :402. */
int pmx_heev_batched(pmx_ctx* ctx, int n, int batch, const double* A, int nev, double* w, double* z);

/* pmx_heev_batched's eigensolver on caller-owned DEVICE buffers; allocates
 * nothing (no cudaMalloc/cudaFree, no allocating library routine), for callers
 * whose device memory is reserved up front by their own pool, or whose
 * latency path must not synchronise the device as cudaMalloc/cudaFree do.
 * A [batch][n][n][2] column-major complex (lower triangle read, overwritten),
 * w [batch][nev], z [batch][nev][n][2] or NULL, info [batch] (0 ok,
 * 1 no convergence, 2 non-finite input): device pointers of the current
 * device. Enqueued on `stream` (a cudaStream_t of the current device; NULL:
 * legacy default stream); returns without waiting for the GPU.
 * Scratch: one fixed 16 MiB device array inside the library (table of at most
 * 1024 matrices, then 4 n nev doubles of inverse-iteration vectors per matrix
 * when z is given). batch > 1024, n > 832, or 32 n nev batch bytes above
 * 16 MiB - 80 KiB (with z) return PMX_ERR_LIMIT. The first call on a device
 * looks the array up (set-up, once per device): make that first call before
 * any stream capture. The address found then is kept for the life of the
 * process, so do not call this entry point again after cudaDeviceReset on
 * that device (the reset makes a new context and the kept address stale).
 * Every call on a device shares the array and rewrites what it reads; calls
 * that overlap on the GPU (different streams or threads) race on it. No
 * counterpart in the reference (added entry point). */
int pmx_heev_batched_noalloc(void* stream, int n, int batch, double* A, int nev, double* w, double* z, int* info);

/* Energy reference: midpoint of eigenvalues nvalence-1 and nvalence at
 * -refpoint (setRefEnergy, src/pmx_epm.cpp:393-428). */
int pmx_ref_energy(pmx_ctx* ctx, const pmx_problem* p, double* offset_eV);

/* Band energies eband [nq][nband] in eV relative to the reference energy
 * (empiricalpseudopotentialmethod, src/pmx_epm.cpp:219-253). */
int pmx_band(pmx_ctx* ctx, const pmx_problem* p, double* eband);

/* ---------------------------------------------------------------- stage 2 */

/* Susceptibility of -switch epsij (chi_tensor, src/pmx_chi.cpp:319-713),
 * epsLL (chi_LL, src/pmx_chi_copy.cpp:320-676) or epsxyz (chi_xyz,
 * src/pmx_chi_copy.cpp:1070-1303, dispatched at src_bkp/pmx.cpp:226-241;
 * spinor eigenvectors always, as the reference), including the Kramers-Kronig
 * step when -kk 1. re/im each hold info.chi_values doubles in .dat order
 * [i][j][q][m][n<=m][f]. precision: PMX_PREC_FP64 or PMX_PREC_MIXED. */
int pmx_chi(pmx_ctx* ctx, const pmx_problem* p, int sw, int precision, double* re, double* im);

/* pmx_chi with the spectra left in device memory: re_dev/im_dev are device
 * pointers with the same layout; epsm_dev (device, [nq][nfreq][2]) receives
 * eps_M of every (q, w) when non-NULL (requires neps <= 64), in which case
 * re_dev and im_dev may both be NULL (eps_M only). */
int pmx_chi_device(pmx_ctx* ctx, const pmx_problem* p, int sw, int precision, double* re_dev, double* im_dev,
                   double* epsm_dev);

/* pmx_chi plus eps_M(q, w) [nq][nfreq][2] of the (L, L) block, as
 * pmx_eps_macroscopic computes it. re and im may both be NULL: eps_M only,
 * chi stays on the device (no copy-out of the 9 blocks). */
int pmx_chi_epsm(pmx_ctx* ctx, const pmx_problem* p, int sw, int precision, double* re, double* im, double* epsm);

/* Macroscopic dielectric function eps_M(q, w) = 1 / [eps^-1]_00 with
 * eps_mn = delta_mn + chi^LL_mn and eps_nm = conj(eps_mn) for n > m, from the
 * (L, L) block of a chi .dat laid out [q][m][n<=m][f] (re and im arrays);
 * epsm [nq][nfreq][2]. Restates the reference's post-processing
 * include/matlab_wrapper/+picomax/+eps/macroscopic.m:13-29, :79 (MATLAB; the
 * C++ reference has no counterpart). neps <= 64. */
int pmx_eps_macroscopic(pmx_ctx* ctx, int neps, int nq, int nfreq, const double* chi_re, const double* chi_im,
                        double* epsm);

/* Electron energy-loss spectrum from eps_M [nq][nfreq][2] (as pmx_chi_epsm
 * returns it): loss [nq][nfreq] = -Im(1 / eps_M(q, w)), and per q the loss
 * peak plasmon [nq][2] = (energy in eV, height): the largest loss at
 * w >= wmin (eV; excludes the low-frequency edge), refined by the vertex of
 * the parabola through the peak and its neighbours. Along a q line (-qpath,
 * or several -qvec) plasmon[:, 0] is the plasmon dispersion. Post-processing
 * of macroscopic.m (include/matlab_wrapper/+picomax/+eps/macroscopic.m:13-29,
 * :79), which computes eps_M; the C++ reference has no counterpart. */
int pmx_eels(pmx_ctx* ctx, int nq, int nfreq, double dfreq, double wmin, const double* epsm, double* loss,
             double* plasmon);

/* ------------------------------------------------------------ k-point grids
 * Symmetry reduction of a Gamma-centred k grid. The reference reads
 * irreducible point lists with weights from files (import_kpt,
 * src/pmx_basis.cpp:200-245; include/kpoints/autoGR and kpLib hold lists made
 * by outside tools) and generates only full grids itself
 * (src/pmx_basis.cpp:256-650).
 *
 * pmx_problem_symmetry (host only): the point-group operations of the
 * problem's Hamiltonian as integer matrices in the reciprocal basis
 * (hkl' = M hkl, reduced k coordinates alike), row-major [nops][9], identity
 * first; ops may be NULL to query nops (at most 96). A lattice operation is
 * kept when, with some translation, the local and spin-orbit form factors of
 * every G difference transform as a potential does and the G list maps onto
 * itself, so that H(k) and H(Rk) have the same spectrum.
 * PMX_KGRID_TIME_REVERSAL adds -M for every M (E(-k) = E(k));
 * PMX_KGRID_LITTLE_GROUP_Q keeps the operations that leave the problem's first
 * q unchanged.
 *
 * pmx_kgrid_reduce (device): the irreducible points of the grid
 * k = sum_j i_j / n_j b_j, 0 <= i_j < n_j, under those operations that map
 * the grid onto itself. nirr receives their count; idx [nirr][3] their grid
 * indices (the smallest linear index i0 + n0 (i1 + n1 i2) of each orbit, in
 * that order) and weight [nirr] the orbit sizes (summing to n0 n1 n2). Pass
 * idx = weight = NULL to query nirr. */
#define PMX_KGRID_TIME_REVERSAL 1
#define PMX_KGRID_LITTLE_GROUP_Q 2
int pmx_problem_symmetry(const pmx_problem* p, int flags, int* nops, int* ops);
int pmx_kgrid_reduce(pmx_ctx* ctx, const pmx_problem* p, const int* n, int flags, int* nirr, int* idx,
                     int* weight);

/* Kramers-Kronig transform of nrows spectra in place, re/im [nrows][nfreq],
 * w_f = dfreq f (kramerskronigtransform, src/pmx_chi.cpp:272-309). */
int pmx_kk(pmx_ctx* ctx, int nrows, int nfreq, double dfreq, double* re, double* im);

/* ---------------------------------------------------------------- batches
 * Several crystals at once. Every eigensolve stage of all problems (reference
 * points, path points, the k and k+q grids of each q) runs as one assembly and
 * one eigensolver launch per matrix-size class (matrices sorted by size),
 * whatever the mix of N_G and SOC; the chi stages that follow run per problem.
 * Results are those of the per-problem calls (same kernels; rounding may
 * differ at the 1e-13 level because the eigensolver schedule can differ).
 * The reference runs one process per crystal. */

/* pmx_band of problems[0..count): eband[i] as pmx_band's output for problems[i]. */
int pmx_band_batch(pmx_ctx* ctx, int count, const pmx_problem* const* problems, double* const* eband);

/* pmx_chi (or pmx_chi_epsm when epsm != NULL and epsm[i] != NULL) of
 * problems[0..count) with one switch and precision; re[i]/im[i] as pmx_chi's
 * outputs for problems[i]. Where eps_M is requested, re and im (the arrays, or
 * both entries i) may be NULL: eps_M only, as for pmx_chi_epsm. Problems are
 * grouped so that the eigenvectors of one group at k and at k+q stay within
 * 2 x 16 GB. */
int pmx_chi_batch(pmx_ctx* ctx, int count, const pmx_problem* const* problems, int sw, int precision,
                  double* const* re, double* const* im, double* const* epsm);

/* ---------------------------------------------------------------- adjoint
 * The reference computes no gradients; these entry points differentiate its
 * band (src/pmx_epm.cpp:56-253) and chi_LL -> eps_M (src/pmx_chi_copy.cpp:
 * 320-676, include/matlab_wrapper/+picomax/+eps/macroscopic.m:13-29) stages
 * with respect to the form factors and SOC parameters, in FP64. */

/* The problem's parameters, in this order: vg[atom][shell] (Ry; the -vg
 * values after the |G|^2 keys), lambda_S (the -uniform_us_so_val value when
 * -use_uniform_us_so is given, else one value per -us_so key in ascending key
 * order), then one lambda_A per -ua_so key (ascending; -ua_so_val_g0 is key 0).
 * values may be NULL to query *count. */
int pmx_problem_params(const pmx_problem* p, double* values, int* count);
/* Replaces the parameters (same order and count) and rebuilds the form-factor
 * tables; the G/k/q tables are unchanged. */
int pmx_problem_set_params(pmx_problem* p, const double* values, int count);

/* Vector-Jacobian product of pmx_band: dE [nq][nband] = dL/d eband,
 * grad [count] = dL/dparams (Hellmann-Feynman, including the reference energy
 * of setRefEnergy, src/pmx_epm.cpp:393-428). */
int pmx_band_vjp(pmx_ctx* ctx, const pmx_problem* p, const double* dE, double* grad);

/* Vector-Jacobian product of eps_M (epsLL, the (L, L) block of chi; NEPS <= 64):
 * deps [nq][nfreq][2] = (dL/dRe eps_M, dL/dIm eps_M), grad [count] = dL/dparams.
 * chi_re/chi_im: the re/im arrays of a FP64 pmx_chi(PMX_SWITCH_EPSLL) call on
 * the same parameters (only their leading (L, L) block is read), or NULL to
 * recompute them. Eigenpairs are recomputed per block of k-points (all
 * eigenvectors of each H(k), for the eigenvector adjoint); eigenvalue pairs
 * closer than 1e-8 eV are treated as degenerate and do not mix. */
int pmx_epsm_vjp(pmx_ctx* ctx, const pmx_problem* p, const double* chi_re, const double* chi_im,
                 const double* deps, double* grad);

/* ---------------------------------------------------------------- driver */

/* The whole picomax program: the reference main (src/pmx.cpp:43-206) plus
 * the epsLL dispatch (src_bkp/pmx.cpp:206-222). Returns the exit code. */
int pmx_main(int argc, const char* const* argv);

#ifdef __cplusplus
}
#endif

#endif /* PICOMAX_B200_H_ */
