// C-ABI of the picomax B200 library (include/picomax.h): problem objects,
// device context, and the host orchestration of the two GPU stages.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/picomax.h"
#include "../cuda/pmx_adjoint.hpp"
#include "../cuda/pmx_chi.hpp"
#include "../cuda/pmx_device.hpp"
#include "../cuda/pmx_mixed.hpp"
#include "pmx_host.hpp"

using pmx::Problem;
using pmx::Vec3;

// ======================================================================= problem
struct pmx_problem {
  Problem p;
  // form-factor tables over hkl differences (see CrystalDev)
  std::vector<double> vloc, vso;  // complex interleaved [side^3][2]
  int soc = 0;
};

namespace {

void build_tables(pmx_problem& P) {
  Problem& p = P.p;
  const int side = 4 * p.imax + 1, off = 2 * p.imax;
  const size_t n3 = (size_t)side * side * side;
  P.vloc.assign(2 * n3, 0.0);
  P.vso.assign(2 * n3, 0.0);
  const Vec3 b1 = p.lat.reciprocal[0], b2 = p.lat.reciprocal[1];
  const Vec3 b3 = p.lat.dim == 3 ? p.lat.reciprocal[2] : Vec3{0, 0, 0};
  P.soc = 0;
  for (int h = -off; h <= off; ++h)
    for (int k = -off; k <= off; ++k)
      for (int l = -off; l <= off; ++l) {
        if (p.lat.dim == 2 && l != 0) continue;
        const Vec3 dG = (double(h) * b1 + double(k) * b2) + double(l) * b3;
        const size_t idx = ((size_t)(h + off) * side + (k + off)) * side + (l + off);
        double re, im;
        pmx::local_potential(p, dG, re, im);
        P.vloc[2 * idx] = re;
        P.vloc[2 * idx + 1] = im;
        pmx::soc_scalar(p, dG, re, im);
        P.vso[2 * idx] = re;
        P.vso[2 * idx + 1] = im;
        if ((h || k || l) && (re != 0.0 || im != 0.0)) P.soc = 1;
      }
}

// SOC current of socCurrent (src/pmx_chi.cpp:203-266) for q = G_m: lambda_S is
// looked up in the -us_so map only, even when -use_uniform_us_so is set.
void soc_current(const Problem& p, const Vec3& q, std::complex<double> out[3]) {
  const std::complex<double> I(0.0, 1.0);
  const double q2 = pmx::sqnorm(q);
  const double la = pmx::soc_form_factor(p.mat.Ua, q2) * pmx::kRy2eV;
  const double ls = pmx::soc_form_factor(p.mat.Us, q2) * pmx::kRy2eV;
  double cs = 0, sn = 0;
  if (p.natom > 0) {
    for (const Vec3& t : p.lat.atomic) {
      cs += std::cos(2.0 * pmx::kPi * pmx::dot(q, t));
      sn += std::sin(2.0 * pmx::kPi * pmx::dot(q, t));
    }
    cs /= p.natom;
    sn /= p.natom;
  }
  const std::complex<double> vso = ls * cs + I * la * sn;
  out[0] = I * vso * (q.y + I * q.z);
  out[1] = I * vso * (q.z - q.x);
  out[2] = I * vso * (-I * q.x - q.y);
}

}  // namespace

extern "C" int pmx_problem_create(int argc, const char* const* argv, pmx_problem** out) {
  if (!out) return PMX_ERR_INVALID;
  *out = nullptr;
  auto P = std::make_unique<pmx_problem>();
  try {
    pmx::build_problem(argc, argv, P->p);
    build_tables(*P);
  } catch (const std::exception& e) {
    std::cerr << "picomax: " << e.what() << std::endl;
    return PMX_ERR_INVALID;
  }
  *out = P.release();
  return PMX_OK;
}

extern "C" void pmx_problem_destroy(pmx_problem* p) { delete p; }

extern "C" int pmx_problem_get_info(const pmx_problem* P, pmx_problem_info* info) {
  if (!P || !info) return PMX_ERR_INVALID;
  const Problem& p = P->p;
  std::memset(info, 0, sizeof(*info));
  info->npw = p.npw();
  info->nh = 2 * p.npw();
  info->soc = P->soc;
  info->neps = p.neps;
  info->nband = p.nband;
  info->nvalence = p.nvalence;
  info->nk = p.nk();
  info->nq = p.nq();
  info->nfreq = p.nfreq;
  info->natom = p.natom;
  info->sw = (int)p.sw;
  info->debug = p.debug;
  info->kk = p.kk;
  info->delta = p.delta;
  info->epsilon = p.epsilon;
  info->dfreq = p.dfreq;
  info->a = p.lat.a;
  info->gcut = p.lat.gcut;
  info->bz_volume = p.lat.bz_volume;
  info->chi_values = 9LL * p.nq() * ((long long)p.neps * (p.neps + 1) / 2) * p.nfreq;
  return PMX_OK;
}

extern "C" int pmx_problem_gvectors(const pmx_problem* P, double* G, int* hkl) {
  if (!P) return PMX_ERR_INVALID;
  for (int i = 0; i < P->p.npw(); ++i)
    for (int x = 0; x < 3; ++x) {
      if (G) G[3 * i + x] = P->p.G[i][x];
      if (hkl) hkl[3 * i + x] = P->p.hkl[i][x];
    }
  return PMX_OK;
}

extern "C" int pmx_problem_loci(const pmx_problem* P, int* loci) {
  if (!P || !loci) return PMX_ERR_INVALID;
  std::copy(P->p.loci.begin(), P->p.loci.end(), loci);
  return PMX_OK;
}

extern "C" int pmx_problem_kpoints(const pmx_problem* P, double* K, double* KW) {
  if (!P) return PMX_ERR_INVALID;
  for (int k = 0; k < P->p.nk(); ++k) {
    if (K)
      for (int x = 0; x < 3; ++x) K[3 * k + x] = P->p.K[k][x];
    if (KW) KW[k] = P->p.KW[k];
  }
  return PMX_OK;
}

extern "C" int pmx_problem_qpoints(const pmx_problem* P, double* Q) {
  if (!P || !Q) return PMX_ERR_INVALID;
  for (int q = 0; q < P->p.nq(); ++q)
    for (int x = 0; x < 3; ++x) Q[3 * q + x] = P->p.lat.Q[q][x];
  return PMX_OK;
}

extern "C" int pmx_problem_dump(const pmx_problem* P, char* buf, size_t len, size_t* needed) {
  if (!P) return PMX_ERR_INVALID;
  std::ostringstream os;
  std::streambuf* old = std::cout.rdbuf(os.rdbuf());
  pmx::print_input(P->p);
  std::cout.rdbuf(old);
  const std::string s = os.str();
  if (needed) *needed = s.size() + 1;
  if (buf && len > 0) {
    const size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return PMX_OK;
}

extern "C" int pmx_problem_write_gpt(const pmx_problem* P) {
  if (!P) return PMX_ERR_INVALID;
  try {
    pmx::write_gpt(P->p);
  } catch (const std::exception& e) {
    std::cerr << "picomax: " << e.what() << std::endl;
    return PMX_ERR_INVALID;
  }
  return PMX_OK;
}

// ======================================================================= context
namespace {

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
  cudaError_t ensure(size_t b) {
    if (b <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&ptr, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(ptr);
  }
};

struct CudaFail : std::runtime_error {
  int code;
  CudaFail(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                                        \
  do {                                                                                               \
    cudaError_t e_ = (x);                                                                            \
    if (e_ != cudaSuccess)                                                                           \
      throw CudaFail(std::string(#x) + ": " + cudaGetErrorString(e_), PMX_ERR_CUDA);                 \
  } while (0)

}  // namespace

struct pmx_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  double stage_ms[5] = {0, 0, 0, 0, 0};
  long long launches = 0;
  long long h2d = 0, d2h = 0;  // bytes copied by the library since creation
  int degenerate_cuts = 0;     // k-points of the last chi call whose NBAND window cut a degenerate set
  int occupation_ties = 0;     // k-points of the last chi call with a window state within 1e-8 eV of E_ref
  // per kernel family: device time (CUDA events around the launches) and launches
  std::map<std::string, std::pair<double, long long>> ktime;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> kpending;
  std::vector<cudaEvent_t> evpool;
  // autotuner: chosen eigensolver schedule per (n, nval, vectors) and the
  // device times measured when it was chosen
  bool autotune = true;
  int fixed_schedule = -1;  // >= 0: this eigensolver schedule on every batch (clamped to the last one)
  long long wait_ns = 0;    // limit of the bounded device waits (0: the kernels' 2 s)
  int fault = 0;            // tests only: injected fault (see pmx_ctx_set_fault)
  int overlap_mode = 1;     // mixed path overlaps: 0 FP64 rounded to FP32, 1 automatic, 2 both (error check),
                            // 3 tensor cores
  std::map<long long, int> heev_choice;
  std::map<long long, std::vector<float>> heev_trials;
  // autotuner of the FP64 overlap kernel's tile shape per (n, npw, largest
  // conduction / valence counts, neps, channels | soc | mode): the shapes tried,
  // their device times, the chosen one
  struct OvlTune {
    int cchunk = 1, vchunk = 1;
    std::vector<int> cc, vc;
    std::vector<float> ms;
  };
  std::map<std::array<int, 6>, OvlTune> ovl_tune;
  // named workspaces
  DevBuf crystal, g, hkl, vloc, vso, items, hbuf, wbuf, zk, zq, scratch, info, rbuf, kgrid;
  DevBuf loci, kpts, uvec, ssoc, qgn, ncd, nvd, cbase, vbase, cidx, vidx, blkoff, dest;
  DevBuf M, dE, wgt, f0, trange, acc, accpv, chi, chi2, mixws, epsm, stats;
  DevBuf t_wk, t_wq, t_kw, t_ntr, t_nblk, t_toff, t_rsrc, t_rde, t_rw, t_rf0, t_cnt, t_sum;  // device transition list
  DevBuf m32, tcerr;  // tensor-core overlaps of the mixed path and their wait status
  // adjoint workspaces
  DevBuf a_chi, a_g, a_gx, a_kk, a_f1, a_f2, a_obar, a_debar, a_mbar, a_zbk, a_zbq, a_lbk, a_lbq;
  DevBuf a_lamk, a_lamq, a_C, a_X, a_R, a_SV, a_SSO, a_kp, a_linv, a_hk, a_trik, a_triq, a_work;
  // several crystals at once (batched entry points)
  DevBuf b_g, b_hkl, b_vloc, b_vso, b_crystal;
  double m2_err = 0.0, m2_max = 0.0;  // |M|^2 error of the mixed path's FP32 overlaps (last call)
  long long mixed_mmas = 0;            // tcgen05 MMA instructions of the mixed contractions so far
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // 0-1 stage timers, 2-3 the autotuner
};

namespace {

struct Timer {
  pmx_ctx* c;
  int slot;
  Timer(pmx_ctx* ctx, int s) : c(ctx), slot(s) { cudaEventRecord(c->ev[0], c->stream); }
  ~Timer() {
    cudaEventRecord(c->ev[1], c->stream);
    cudaEventSynchronize(c->ev[1]);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stage_ms[slot] += ms;
  }
};

// Brackets the launches of one kernel family with CUDA events on the context
// stream; durations are collected when the stream is next synchronised.
struct KTime {
  pmx_ctx* c;
  std::string name;
  cudaEvent_t a, b;
  KTime(pmx_ctx* ctx, const char* n) : c(ctx), name(n) {
    a = take();
    b = take();
    cudaEventRecord(a, c->stream);
  }
  cudaEvent_t take() {
    if (!c->evpool.empty()) {
      cudaEvent_t e = c->evpool.back();
      c->evpool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  ~KTime() {
    cudaEventRecord(b, c->stream);
    c->kpending.push_back({name, {a, b}});
  }
};

void collect_ktimes(pmx_ctx* c) {
  for (auto& kp : c->kpending) {
    float ms = 0;
    if (cudaEventSynchronize(kp.second.second) == cudaSuccess &&
        cudaEventElapsedTime(&ms, kp.second.first, kp.second.second) == cudaSuccess) {
      auto& t = c->ktime[kp.first];
      t.first += ms;
      t.second += 1;
    }
    c->evpool.push_back(kp.second.first);
    c->evpool.push_back(kp.second.second);
  }
  c->kpending.clear();
}

template <class F>
int guarded(pmx_ctx* ctx, F&& f) {
  if (!ctx) return PMX_ERR_INVALID;
  ctx->err.clear();
  try {
    CK(cudaSetDevice(ctx->device));
    const int rc = f();
    collect_ktimes(ctx);
    return rc;
  } catch (const CudaFail& e) {
    ctx->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return PMX_ERR_INVALID;
  }
}

void h2d(pmx_ctx* c, DevBuf& b, const void* src, size_t bytes) {
  CK(b.ensure(std::max<size_t>(bytes, 16)));
  if (bytes) CK(cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, c->stream));
  c->h2d += (long long)bytes;
}

// The crystal as the kernels see it, uploaded into the context.
struct DevCrystal {
  pmx::dev::CrystalDev host;
  pmx::dev::CrystalDev* dev = nullptr;
  int soc = 0;
  int npw = 0;
  int n = 0;        // eigenproblem dimension
};

DevCrystal upload_crystal(pmx_ctx* c, const pmx_problem* P, int force_spinor) {
  const Problem& p = P->p;
  DevCrystal d;
  d.npw = p.npw();
  d.soc = (P->soc || force_spinor) ? 1 : 0;
  d.n = d.soc ? 2 * d.npw : d.npw;
  std::vector<double> G(3 * d.npw);
  std::vector<int> H(3 * d.npw);
  for (int i = 0; i < d.npw; ++i)
    for (int x = 0; x < 3; ++x) {
      G[3 * i + x] = p.G[i][x];
      H[3 * i + x] = p.hkl[i][x];
    }
  h2d(c, c->g, G.data(), G.size() * sizeof(double));
  h2d(c, c->hkl, H.data(), H.size() * sizeof(int));
  h2d(c, c->vloc, P->vloc.data(), P->vloc.size() * sizeof(double));
  h2d(c, c->vso, P->vso.data(), P->vso.size() * sizeof(double));
  pmx::dev::CrystalDev& cd = d.host;
  cd.npw = d.npw;
  cd.soc = d.soc;
  cd.imax = p.imax;
  cd.side = 4 * p.imax + 1;
  const double s = 2.0 * pmx::kPi / p.lat.a;
  cd.kin = pmx::kKCON * (s * s);
  cd.G = c->g.as<double>();
  cd.hkl = c->hkl.as<int>();
  cd.vloc = c->vloc.as<double2>();
  cd.vso = c->vso.as<double2>();
  h2d(c, c->crystal, &cd, sizeof(cd));
  d.dev = c->crystal.as<pmx::dev::CrystalDev>();
  return d;
}

// Eigensolver dispatch. Where the two-stage solver applies (matrices too
// large for the shared-memory-resident one-stage kernel, padded size <= 832,
// and no export of the one-stage reduction for the adjoint) it is schedule 0
// and the one-stage schedules follow; otherwise only the one-stage schedules
// are offered. A launch's items then carry the padded leading dimension and
// a slot of the band reflector buffer (ctx rbuf).
bool use_two_stage(int max_n, bool tri) {
  return !tri && max_n > pmx::dev::heev_smem_max_n() && pmx::dev::heev2_supported(max_n);
}
int eig_variants(int max_n, int max_nval, bool tri) {
  return (use_two_stage(max_n, tri) ? 1 : 0) + pmx::dev::heev_variants(max_n, max_nval);
}
// leading dimension / reflector slot (double2) of an item of size n in a
// launch whose largest matrix is max_n
int eig_ld(int n, int max_n, bool tri) { return use_two_stage(max_n, tri) ? pmx::dev::heev2_ld(n) : n; }
size_t eig_rstride(int n, int max_n, bool tri) {
  return use_two_stage(max_n, tri) ? pmx::dev::heev2_rbuf_double2(pmx::dev::heev2_ld(n), pmx::dev::heev2_ld(max_n))
                                    : 0;
}
// the context's wait limit and test fault hooks on an eigensolver item
void eig_hooks(const pmx_ctx* c, pmx::dev::EigItem& it) {
  it.bisect_cap = c->fault == 2 ? 1 : 0;
  it.wait_ns = c->wait_ns;
  it.wait_fault = c->fault == 3 ? 1 : 0;
}
// status of a failed eigensolve: 3 = a bounded wait of the bulge chase gave up
int eig_status_error(int status) { return status == 3 ? PMX_ERR_TIMEOUT : PMX_ERR_NOCONV; }
cudaError_t eig_launch(pmx_ctx* c, const pmx::dev::EigItem* items, int nitems, int max_n, int max_nval,
                       int max_nvec, double2* hbuf, double* wbuf, double2* zbuf, double* scratch, int* info,
                       int variant, double* tri = nullptr) {
  if (use_two_stage(max_n, tri != nullptr)) {
    if (variant == 0)
      return pmx::dev::launch_heev2(items, nitems, max_n, max_nval, max_nvec, hbuf, wbuf, zbuf, scratch,
                                    c->rbuf.as<double2>(), info, c->stream);
    variant -= 1;
  }
  return pmx::dev::launch_heev(items, nitems, max_n, max_nval, hbuf, wbuf, zbuf, scratch, info, c->stream, variant,
                               tri);
}

// H workspace of one chunk of eigensolves: 2 GB, or up to 8 GB where two
// waves of 148 matrices of the largest size need more (n > 832), so that the
// large sizes still fill the GPU; 2 GB with the tridiagonal export, whose
// callers keep their k-points within one chunk of that size
size_t h_budget(size_t hbytes_max, bool tri) {
  const size_t base = (size_t)2 << 30;
  return tri ? base : std::max(base, std::min((size_t)8 << 30, 296 * hbytes_max));
}

// Assembles and diagonalises H(k) for every k; the lowest nval eigenvalues
// go to w (host, [nk][nval]); with zdev the lowest nvec eigenvectors go to
// zdev ([nk][nvec][n]).
// With tri (device, [nk][4 n]) the tridiagonal form of every H(k) is exported
// and the reflectors of the last chunk stay in c->hbuf (ks must then fit one
// chunk: nk <= 2 GB / (16 n^2)).
void solve_k(pmx_ctx* c, const DevCrystal& dc, const std::vector<Vec3>& ks, int nval, int nvec, double2* zdev,
             std::vector<double>& w, double* tri = nullptr) {
  const int nk = (int)ks.size(), n = dc.n;
  w.assign((size_t)nk * nval, 0.0);
  if (nk == 0) return;
  if (nval > n) throw CudaFail("too many eigenvalues requested", PMX_ERR_INVALID);
  const bool vec = zdev != nullptr && nvec > 0;
  const bool tri_req = tri != nullptr;
  const int ld = eig_ld(n, n, tri_req);
  const size_t hbytes = (size_t)ld * ld * sizeof(double2);
  int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nk, h_budget(hbytes, tri_req) / hbytes));
  chunk = std::min(chunk, 4096);
  if (nk > chunk) {  // several chunks: each a whole number of waves of CTAs
    const int unit = pmx::dev::heev_batch_unit(n, nval);
    if (chunk >= unit) chunk = chunk / unit * unit;
  }
  CK(c->hbuf.ensure(hbytes * chunk));
  CK(c->wbuf.ensure(sizeof(double) * (size_t)nk * nval));
  const size_t sstride = pmx::dev::heev_scratch_doubles(n, vec ? nvec : 0, n);
  const bool per_item = vec || n > 832;  // without vectors the scratch holds only the large-n partial sums
  CK(c->scratch.ensure(sizeof(double) * sstride * (per_item ? chunk : 1)));
  CK(c->info.ensure(sizeof(int) * chunk));
  const size_t rstride = eig_rstride(n, n, tri_req);
  if (rstride) CK(c->rbuf.ensure(sizeof(double2) * rstride * chunk));
  std::vector<pmx::dev::EigItem> items(chunk);
  std::vector<int> info(chunk);
  for (int k0 = 0; k0 < nk; k0 += chunk) {
    const int cnt = std::min(chunk, nk - k0);
    for (int i = 0; i < cnt; ++i) {
      pmx::dev::EigItem& it = items[i];
      it = pmx::dev::EigItem{};
      it.crystal = 0;
      it.n = n;
      it.nev = vec ? nvec : 0;
      it.nval = nval;
      it.want_vec = vec ? 1 : 0;
      for (int x = 0; x < 3; ++x) it.k[x] = ks[k0 + i][x];
      it.h_off = (long long)i * ld * ld;
      it.w_off = (long long)(k0 + i) * nval;
      it.z_off = (long long)(k0 + i) * nvec * n;
      it.s_off = per_item ? (long long)(i * sstride) : 0;
      it.ld = ld;
      it.r_off = (long long)(i * rstride);
      eig_hooks(c, it);
    }
    h2d(c, c->items, items.data(), sizeof(pmx::dev::EigItem) * cnt);
    {
      KTime kt(c, "assemble");
      CK(pmx::dev::launch_assemble(dc.dev, c->items.as<pmx::dev::EigItem>(), cnt, dc.npw, c->hbuf.as<double2>(),
                                   c->stream));
    }
    // eigensolver schedule: cached choice, or timed once on the first large
    // enough chunk (every candidate runs on that chunk; the chosen one runs
    // last so the results come from it)
    const long long key = ((long long)n * 1024 + nval) * 2 + (vec ? 1 : 0);
    int variant = 0;
    const int nvar = eig_variants(n, nval, tri_req);
    auto it_choice = c->heev_choice.find(key);
    if (c->fixed_schedule >= 0) {
      variant = std::min(c->fixed_schedule, nvar - 1);
    } else if (it_choice != c->heev_choice.end()) {
      variant = it_choice->second;
    } else if (nvar > 1 && c->autotune && cnt >= 148) {
      std::vector<float> ms(nvar, 0.f);
      for (int v = 0; v < nvar; ++v) {
        CK(cudaEventRecord(c->ev[2], c->stream));
        CK(eig_launch(c, c->items.as<pmx::dev::EigItem>(), cnt, n, nval, vec ? nvec : 0, c->hbuf.as<double2>(),
                      c->wbuf.as<double>(), vec ? zdev : c->hbuf.as<double2>(), c->scratch.as<double>(),
                      c->info.as<int>(), v));
        CK(cudaEventRecord(c->ev[3], c->stream));
        CK(cudaEventSynchronize(c->ev[3]));
        CK(cudaEventElapsedTime(&ms[v], c->ev[2], c->ev[3]));
        c->launches += 1;
        // H is overwritten by the reduction: rebuild it for the next candidate
        CK(pmx::dev::launch_assemble(dc.dev, c->items.as<pmx::dev::EigItem>(), cnt, dc.npw, c->hbuf.as<double2>(),
                                     c->stream));
        c->launches += 1;
      }
      variant = (int)(std::min_element(ms.begin(), ms.end()) - ms.begin());
      c->heev_choice[key] = variant;
      c->heev_trials[key] = ms;
    }
    {
      KTime kt(c, "heev");
      CK(eig_launch(c, c->items.as<pmx::dev::EigItem>(), cnt, n, nval, vec ? nvec : 0, c->hbuf.as<double2>(),
                    c->wbuf.as<double>(), vec ? zdev : c->hbuf.as<double2>(), c->scratch.as<double>(),
                    c->info.as<int>(), variant, tri ? tri + (size_t)k0 * 4 * n : nullptr));
    }
    c->launches += 2;
    CK(cudaMemcpyAsync(info.data(), c->info.ptr, sizeof(int) * cnt, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->d2h += sizeof(int) * cnt;
    for (int i = 0; i < cnt; ++i)
      if (info[i] != 0)
        throw CudaFail("eigensolver failed (status " + std::to_string(info[i]) + ") at k-point " +
                           std::to_string(k0 + i),
                       eig_status_error(info[i]));
  }
  CK(cudaMemcpyAsync(w.data(), c->wbuf.ptr, sizeof(double) * w.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->d2h += sizeof(double) * w.size();
}

// Spinor eigenvalue s of a solved item (spatial spectrum doubled without SOC).
inline double spinor_eig(const std::vector<double>& w, int nev, int k, int s, int soc) {
  return soc ? w[(size_t)k * nev + s] : w[(size_t)k * nev + s / 2];
}

// Number of solved states needed to cover `spinor` spinor states.
inline int solved_states(int spinor, int soc) { return soc ? spinor : (spinor + 1) / 2; }

double ref_energy(pmx_ctx* c, const pmx_problem* P, const DevCrystal& dc) {
  const Problem& p = P->p;
  const int nh = 2 * p.npw();
  if (!(p.nvalence > 0 && p.nvalence < nh)) {
    std::cout << "WARNING::setRefEnergy:: nvalence is out of bounds for eigenvalues. Setting offset to 0."
              << std::endl;
    return 0.0;
  }
  const int nev = solved_states(p.nvalence + 1, dc.soc);
  std::vector<double> w;
  solve_k(c, dc, {p.refpoint}, nev, 0, nullptr, w);
  return (spinor_eig(w, nev, 0, p.nvalence - 1, dc.soc) + spinor_eig(w, nev, 0, p.nvalence, dc.soc)) / 2.0;
}

}  // namespace

extern "C" int pmx_ctx_create(int device, pmx_ctx** out) {
  if (!out) return PMX_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return PMX_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return PMX_ERR_INVALID;
  auto c = std::make_unique<pmx_ctx>();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return PMX_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return PMX_ERR_CUDA;
  for (auto& e : c->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return PMX_ERR_CUDA;
  *out = c.release();
  return PMX_OK;
}

extern "C" void pmx_ctx_destroy(pmx_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& kp : c->kpending) {
    cudaEventDestroy(kp.second.first);
    cudaEventDestroy(kp.second.second);
  }
  for (auto& e : c->evpool) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" const char* pmx_ctx_last_error(const pmx_ctx* c) { return c ? c->err.c_str() : "null context"; }

extern "C" int pmx_ctx_stage_times(const pmx_ctx* c, double* ms5) {
  if (!c || !ms5) return PMX_ERR_INVALID;
  for (int i = 0; i < 5; ++i) ms5[i] = c->stage_ms[i];
  return PMX_OK;
}

extern "C" long long pmx_ctx_kernel_launches(const pmx_ctx* c) { return c ? c->launches : -1; }

// ======================================================================= stage 1
extern "C" int pmx_hamiltonian(pmx_ctx* ctx, const pmx_problem* P, const double* kpts, int nk, double* out) {
  if (!P || (nk > 0 && (!kpts || !out)) || nk < 0) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    DevCrystal dc = upload_crystal(ctx, P, 1);
    const int n = dc.n;
    std::vector<pmx::dev::EigItem> items(nk);
    for (int i = 0; i < nk; ++i) {
      items[i].crystal = 0;
      items[i].n = n;
      for (int x = 0; x < 3; ++x) items[i].k[x] = kpts[3 * i + x];
      items[i].h_off = (long long)i * n * n;
    }
    const size_t bytes = sizeof(double2) * (size_t)n * n * nk;
    CK(ctx->hbuf.ensure(std::max<size_t>(bytes, 16)));
    h2d(ctx, ctx->items, items.data(), sizeof(pmx::dev::EigItem) * nk);
    CK(pmx::dev::launch_assemble(dc.dev, ctx->items.as<pmx::dev::EigItem>(), nk, dc.npw, ctx->hbuf.as<double2>(),
                                 ctx->stream));
    ctx->launches += 1;
    CK(cudaMemcpyAsync(out, ctx->hbuf.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return (int)PMX_OK;
  });
}

extern "C" int pmx_heev_batched(pmx_ctx* ctx, int n, int batch, const double* A, int nev, double* w, double* z) {
  if (n <= 0 || batch < 0 || nev <= 0 || nev > n || (batch > 0 && (!A || !w))) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    const int ld = eig_ld(n, n, false);
    const size_t hb = sizeof(double2) * (size_t)ld * ld;
    CK(ctx->hbuf.ensure(std::max<size_t>(hb * batch, 16)));
    const size_t rstride = eig_rstride(n, n, false);
    if (rstride) CK(ctx->rbuf.ensure(sizeof(double2) * rstride * std::max(batch, 1)));
    CK(ctx->wbuf.ensure(std::max<size_t>(sizeof(double) * (size_t)batch * nev, 16)));
    CK(ctx->zk.ensure(std::max<size_t>(sizeof(double2) * (size_t)batch * nev * n, 16)));
    const size_t sstride = pmx::dev::heev_scratch_doubles(n, z ? nev : 0, n);
    CK(ctx->scratch.ensure(std::max<size_t>(sizeof(double) * sstride * batch, 16)));
    CK(ctx->info.ensure(std::max<size_t>(sizeof(int) * batch, 16)));
    std::vector<pmx::dev::EigItem> items(batch);
    for (int i = 0; i < batch; ++i) {
      items[i] = pmx::dev::EigItem{};
      items[i].n = n;
      items[i].nev = z ? nev : 0;
      items[i].nval = nev;
      items[i].want_vec = z ? 1 : 0;
      items[i].h_off = (long long)i * ld * ld;
      items[i].w_off = (long long)i * nev;
      items[i].z_off = (long long)i * nev * n;
      items[i].s_off = (long long)(i * sstride);
      items[i].ld = ld;
      items[i].r_off = (long long)(i * rstride);
      eig_hooks(ctx, items[i]);
    }
    if (batch == 0) return (int)PMX_OK;
    if (ld == n) {
      CK(cudaMemcpyAsync(ctx->hbuf.ptr, A, hb * batch, cudaMemcpyHostToDevice, ctx->stream));
    } else {  // columns of n into the zero-padded ld x ld layout
      CK(cudaMemsetAsync(ctx->hbuf.ptr, 0, hb * batch, ctx->stream));
      for (int i = 0; i < batch; ++i)
        CK(cudaMemcpy2DAsync(ctx->hbuf.as<double2>() + (size_t)i * ld * ld, sizeof(double2) * ld,
                             A + (size_t)2 * i * n * n, sizeof(double2) * n, sizeof(double2) * n, n,
                             cudaMemcpyHostToDevice, ctx->stream));
    }
    h2d(ctx, ctx->items, items.data(), sizeof(pmx::dev::EigItem) * batch);
    {
      KTime kt(ctx, "heev");
      CK(eig_launch(ctx, ctx->items.as<pmx::dev::EigItem>(), batch, n, nev, z ? nev : 0, ctx->hbuf.as<double2>(),
                    ctx->wbuf.as<double>(), ctx->zk.as<double2>(), ctx->scratch.as<double>(), ctx->info.as<int>(),
                    std::min(std::max(ctx->fixed_schedule, 0), eig_variants(n, nev, false) - 1)));
    }
    ctx->launches += 1;
    std::vector<int> info(batch);
    CK(cudaMemcpyAsync(info.data(), ctx->info.ptr, sizeof(int) * batch, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(w, ctx->wbuf.ptr, sizeof(double) * batch * nev, cudaMemcpyDeviceToHost, ctx->stream));
    if (z)
      CK(cudaMemcpyAsync(z, ctx->zk.ptr, sizeof(double2) * (size_t)batch * nev * n, cudaMemcpyDeviceToHost,
                         ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < batch; ++i)
      if (info[i])
        throw CudaFail("eigensolver failed (status " + std::to_string(info[i]) + ") for matrix " + std::to_string(i),
                       eig_status_error(info[i]));
    return (int)PMX_OK;
  });
}

extern "C" int pmx_ref_energy(pmx_ctx* ctx, const pmx_problem* P, double* off) {
  if (!P || !off) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    DevCrystal dc = upload_crystal(ctx, P, 0);
    *off = ref_energy(ctx, P, dc);
    return (int)PMX_OK;
  });
}

extern "C" int pmx_band(pmx_ctx* ctx, const pmx_problem* P, double* eband) {
  if (!P || (!eband && P->p.nq() > 0)) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    const Problem& p = P->p;
    for (double& t : ctx->stage_ms) t = 0;
    Timer tm(ctx, 0);
    DevCrystal dc = upload_crystal(ctx, P, 0);
    const double off = ref_energy(ctx, P, dc);
    const int nh = 2 * p.npw();
    const int nkeep = std::min(p.nband, nh);
    if (nkeep <= 0) {
      std::fill(eband, eband + (size_t)p.nq() * std::max(p.nband, 0), 0.0);
      return (int)PMX_OK;
    }
    const int nev = solved_states(nkeep, dc.soc);
    std::vector<double> w;
    solve_k(ctx, dc, p.lat.Q, nev, 0, nullptr, w);
    for (int q = 0; q < p.nq(); ++q)
      for (int n = 0; n < p.nband; ++n)
        eband[(size_t)q * p.nband + n] = n < nh ? spinor_eig(w, nev, q, n, dc.soc) - off : 0.0;
    return (int)PMX_OK;
  });
}

// ======================================================================= stage 2
namespace {

struct Transitions {
  std::vector<int> ncd, nvd, cbase, vbase, cidx, vidx;
  std::vector<long long> blkoff, dest;
  std::vector<double> dE, wgt;
  std::vector<int> f0;
  long long T = 0;
};

// Occupations and transition list of one q (src/pmx_chi.cpp:391-397, :477-483):
// conduction states are counted down from the top of the NBAND window while
// E - E_ref > 0, valence states up from the bottom while E - E_ref <= 0.
// wk/wq hold nval eigenvalues per k (spatial states without SOC). `cuts`
// counts k and k+q points where state NBAND-1 and NBAND are degenerate.
// k0/k1 restrict the list to k-points [k0, k1) (wk/wq and the per-k arrays
// then count from k0).
// The result lives in a per-thread buffer that the next call on the thread
// rebuilds in place (large vectors freed and allocated every call would be
// paged in again each time).
const Transitions& build_transitions(const Problem& p, int soc, int nval, const std::vector<double>& wk,
                              const std::vector<double>& wq, double off, bool sort_by_window, int& cuts,
                              int k0 = 0, int k1 = -1, int* ties = nullptr, bool xyz = false) {
  static thread_local Transitions T;
  T.T = 0;
  T.cidx.clear();
  T.vidx.clear();
  if (k1 < 0) k1 = p.nk();
  const int nk = k1 - k0, NB = p.nband;
  T.ncd.resize(nk);
  T.nvd.resize(nk);
  T.cbase.resize(nk);
  T.vbase.resize(nk);
  T.blkoff.resize(nk);
  struct Raw {
    long long src;
    double dE, w;
    int f0;
  };
  // kept across calls: the list is rebuilt for every q and reused in place
  static thread_local std::vector<Raw> raw;
  raw.clear();
  raw.reserve((size_t)nk * (size_t)(NB / 2 + 1) * (size_t)(NB / 2 + 1));
  T.cidx.reserve((size_t)nk * NB);
  T.vidx.reserve((size_t)nk * NB);
  long long blk = 0;
  const double df = p.dfreq, w0 = p.freq.empty() ? 0.0 : p.freq[0];
  const int nh = 2 * p.npw();
  std::vector<int> cs, vs;  // distinct solved conduction / valence states of a k-point
  cs.reserve(NB);
  vs.reserve(NB);
  for (int k = 0; k < nk; ++k) {
    const int kg = k0 + k;  // global k index
    if (NB < nh) {
      const bool cut_k = std::abs(spinor_eig(wk, nval, k, NB, soc) - spinor_eig(wk, nval, k, NB - 1, soc)) < 1e-8;
      const bool cut_q = std::abs(spinor_eig(wq, nval, k, NB, soc) - spinor_eig(wq, nval, k, NB - 1, soc)) < 1e-8;
      cuts += (int)cut_k + (int)cut_q;
    }
    if (ties) {
      // a state of the window within 1e-8 eV of E_ref: its occupation is decided by rounding
      bool tk = false, tq = false;
      for (int s = 0; s < NB && s < nh; ++s) {
        tk |= std::abs(spinor_eig(wk, nval, k, s, soc) - off) < 1e-8;
        tq |= std::abs(spinor_eig(wq, nval, k, s, soc) - off) < 1e-8;
      }
      *ties += (int)tk + (int)tq;
    }
    int nc = 0, nv = 0;
    if (xyz) {
      // chi_xyz (src/pmx_chi_copy.cpp:1128-1140, :1178-1186): the conjugated
      // (first) set is the valence at k, counted up while E - E_ref <= 0; the
      // second set the conduction at k+q, counted down from the top while > 0.
      // Spinor states only.
      std::vector<int> fs, ss;
      while (nc < NB && spinor_eig(wk, nval, k, nc, soc) - off <= 0) fs.push_back(nc++);
      while (nv < NB && spinor_eig(wq, nval, k, NB - 1 - nv, soc) - off > 0) ss.push_back(NB - 1 - nv++);
      T.ncd[k] = (int)fs.size();
      T.nvd[k] = (int)ss.size();
      T.cbase[k] = (int)T.cidx.size();
      T.vbase[k] = (int)T.vidx.size();
      T.cidx.insert(T.cidx.end(), fs.begin(), fs.end());
      T.vidx.insert(T.vidx.end(), ss.begin(), ss.end());
      T.blkoff[k] = blk;
      for (size_t a = 0; a < fs.size(); ++a)
        for (size_t b = 0; b < ss.size(); ++b) {
          const double de = (spinor_eig(wq, nval, k, ss[b], soc) - off) - (spinor_eig(wk, nval, k, fs[a], soc) - off);
          raw.push_back({blk + (long long)(a * ss.size() + b), de, p.KW[kg], (int)((de - w0) / df)});
        }
      blk += (long long)fs.size() * ss.size();
      continue;
    }
    while (nc < NB && spinor_eig(wk, nval, k, NB - 1 - nc, soc) - off > 0) ++nc;
    while (nv < NB && spinor_eig(wq, nval, k, nv, soc) - off <= 0) ++nv;
    // distinct solved states
    cs.clear();
    vs.clear();
    for (int c = 0; c < nc; ++c) {
      const int st = soc ? NB - 1 - c : (NB - 1 - c) / 2;
      if (cs.empty() || cs.back() != st) cs.push_back(st);
    }
    for (int v = 0; v < nv; ++v) {
      const int st = soc ? v : v / 2;
      if (vs.empty() || vs.back() != st) vs.push_back(st);
    }
    T.ncd[k] = (int)cs.size();
    T.nvd[k] = (int)vs.size();
    T.cbase[k] = (int)T.cidx.size();
    T.vbase[k] = (int)T.vidx.size();
    T.cidx.insert(T.cidx.end(), cs.begin(), cs.end());
    T.vidx.insert(T.vidx.end(), vs.begin(), vs.end());
    T.blkoff[k] = blk;
    for (size_t ic = 0; ic < cs.size(); ++ic)
      for (size_t iv = 0; iv < vs.size(); ++iv) {
        int mult = 1;
        if (!soc) {
          // spin copies (2 st + sigma) present on both sides with equal spin
          mult = 0;
          for (int sg = 0; sg < 2; ++sg) {
            const int sc = 2 * cs[ic] + sg, sv = 2 * vs[iv] + sg;
            const int c = NB - 1 - sc;
            if (sc <= NB - 1 && c >= 0 && c < nc && sv < nv) ++mult;
          }
        }
        const long long src = blk + (long long)ic * vs.size() + iv;
        if (mult == 0) continue;
        const int s_c = soc ? cs[ic] : 2 * cs[ic];
        const int s_v = soc ? vs[iv] : 2 * vs[iv];
        const double ec = spinor_eig(wk, nval, k, s_c, soc) - off;
        const double ev = spinor_eig(wq, nval, k, s_v, soc) - off;
        const double de = ec - ev;
        raw.push_back({src, de, p.KW[kg] * mult, (int)((de - w0) / df)});
      }
    blk += (long long)cs.size() * vs.size();
  }
  // transition t of the output: raw entries in k order, stably sorted by
  // window start when asked (a counting sort over the f0 range, a few
  // thousand frequencies, scattering straight into the output arrays; the
  // comparison sort only for an unusual range)
  T.T = (long long)raw.size();
  T.dest.assign(std::max<long long>(blk, 1), -1);
  T.dE.resize(raw.size());
  T.wgt.resize(raw.size());
  T.f0.resize(raw.size());
  // plain pointers: the worker threads below must not name this thread's
  // thread_local buffers (each thread has its own)
  long long* o_dest = T.dest.data();
  double* o_dE = T.dE.data();
  double* o_wgt = T.wgt.data();
  int* o_f0 = T.f0.data();
  const Raw* in = raw.data();
  auto put = [=](size_t t, const Raw& r) {
    o_dest[r.src] = (long long)t;
    o_dE[t] = r.dE;
    o_wgt[t] = r.w;
    o_f0[t] = r.f0;
  };
  int lo = 0, hi = 0;
  if (!raw.empty()) {
    lo = hi = raw[0].f0;
    for (const Raw& r : raw) {
      lo = std::min(lo, r.f0);
      hi = std::max(hi, r.f0);
    }
  }
  if (!sort_by_window || raw.empty()) {
    for (size_t t = 0; t < raw.size(); ++t) put(t, raw[t]);
  } else if ((long long)hi - lo < (1LL << 24)) {
    // parallel stable counting sort: contiguous parts of the k-ordered list,
    // one histogram per part; bucket b of part j starts after bucket b of
    // parts < j and after all smaller buckets, so the order is the serial one
    const size_t nb = (size_t)(hi - lo) + 1, nr = raw.size();
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int parts = (int)std::min<size_t>(std::min<unsigned>(hw, 16u), std::max<size_t>(1, nr / 32768));
    std::vector<std::vector<long long>> cnt(parts, std::vector<long long>(nb, 0));
    auto range = [&](int j) { return std::make_pair(nr * j / parts, nr * (j + 1) / parts); };
    auto run = [&](auto&& fn) {
      std::vector<std::thread> th;
      for (int j = 1; j < parts; ++j) th.emplace_back(fn, j);
      fn(0);
      for (auto& t : th) t.join();
    };
    run([&](int j) {
      const auto rg = range(j);
      for (size_t t = rg.first; t < rg.second; ++t) ++cnt[j][(size_t)(in[t].f0 - lo)];
    });
    long long acc = 0;
    for (size_t b = 0; b < nb; ++b)
      for (int j = 0; j < parts; ++j) {
        const long long c = cnt[j][b];
        cnt[j][b] = acc;
        acc += c;
      }
    run([&](int j) {
      const auto rg = range(j);
      std::vector<long long>& pos = cnt[j];
      for (size_t t = rg.first; t < rg.second; ++t) put((size_t)pos[(size_t)(in[t].f0 - lo)]++, in[t]);
    });
  } else {
    std::stable_sort(raw.begin(), raw.end(), [](const Raw& a, const Raw& b) { return a.f0 < b.f0; });
    for (size_t t = 0; t < raw.size(); ++t) put(t, raw[t]);
  }
  return T;
}

int window_half(const Problem& p) {
  const double df = p.dfreq;
  const int g = std::max(1, int(6.0 * p.epsilon / df));
  const int l = std::max(1, int(50.0 * p.epsilon / df));
  return p.delta == 1 ? l : g;
}

}  // namespace

namespace {

// Per-problem constants of the chi stage.
struct ChiPlan {
  int mode, nk, nq, neps, nf, np, nev, nval, n, nch, W, FT, nft;
  size_t blkvals;  // one q, one of Re/Im
  bool pv;
  pmx::dev::ScaleArgs sa;
};

ChiPlan chi_plan(const Problem& p, int sw, const DevCrystal& dc) {
  if (!p.have_freq || p.nfreq <= 0 || !(p.dfreq > 0))
    throw std::runtime_error("-nfreq and -dfreq are required for the chi switches");
  if (p.nband > 2 * p.npw()) throw std::runtime_error("-nband exceeds the Hamiltonian dimension");
  if (p.nband <= 0) throw std::runtime_error("-nband must be positive");
  ChiPlan pl;
  pl.mode = sw == PMX_SWITCH_EPSLL ? 1 : (sw == PMX_SWITCH_EPSXYZ ? 2 : 0);
  if (pl.mode == 2 && !dc.soc) throw std::runtime_error("epsxyz needs the spinor eigenproblem");
  pl.nk = p.nk();
  pl.nq = p.nq();
  pl.neps = p.neps;
  pl.nf = p.nfreq;
  pl.np = pl.neps * (pl.neps + 1) / 2;
  pl.blkvals = (size_t)9 * pl.np * pl.nf;
  pl.nev = solved_states(p.nband, dc.soc);
  pl.nval = std::min(solved_states(p.nband + 1, dc.soc), dc.n);
  pl.n = dc.n;
  pl.nch = (pl.mode == 0 && dc.soc) ? 4 : 1;
  // scale factors (src/pmx_chi.cpp:341, src/pmx_chi_copy.cpp:351-360)
  const double a_cm = p.lat.a * pmx::kAngstrom, bz = p.lat.bz_volume;
  pmx::dev::ScaleArgs& sa = pl.sa;
  sa = pmx::dev::ScaleArgs{};
  sa.mode = pl.mode;
  sa.np = pl.np;
  sa.nf = pl.nf;
  sa.dfreq = p.dfreq;
  sa.sf = 4.0 * bz * std::pow(pmx::kPi, 5) * std::pow(pmx::kHbar, 4) * std::pow(pmx::kE, 2) /
          (std::pow(pmx::kEV, 3) * std::pow(pmx::kEm, 2) * std::pow(a_cm, 5));
  sa.sf_ll = 2.0 * bz * std::pow(pmx::kE, 2) / (pmx::kPi * pmx::kEV * a_cm);
  sa.sf_tt = 32.0 * bz * std::pow(pmx::kPi, 3) * std::pow(pmx::kHbar, 4) * std::pow(pmx::kE, 2) /
             (std::pow(pmx::kEV, 3) * std::pow(pmx::kEm, 2) * std::pow(a_cm, 5));
  sa.sf_lt = 8.0 * bz * pmx::kPi * std::pow(pmx::kHbar, 2) * std::pow(pmx::kE, 2) /
             (std::pow(pmx::kEV, 2) * pmx::kEm * std::pow(a_cm, 3));
  pl.W = pl.mode == 0 ? window_half(p) : -1;
  pl.FT = pmx::dev::contract_ftile();
  pl.nft = (pl.nf + pl.FT - 1) / pl.FT;
  pl.pv = pl.mode >= 1 && p.kk == 0;
  return pl;
}

void chi_buffers(pmx_ctx* ctx, const ChiPlan& pl) {
  CK(ctx->acc.ensure(sizeof(double) * 2 * pl.blkvals));
  CK(ctx->chi.ensure(sizeof(double) * 2 * pl.blkvals));
  CK(ctx->chi2.ensure(sizeof(double) * 2 * pl.blkvals));
  if (pl.pv) CK(ctx->accpv.ensure(sizeof(double) * 2 * pl.blkvals));
}

// Static tables of one problem's chi stage (loci, k-points).
void chi_tables(pmx_ctx* ctx, const Problem& p) {
  h2d(ctx, ctx->loci, p.loci.data(), sizeof(int) * p.loci.size());
  std::vector<double> kp(3 * (size_t)p.nk());
  for (int k = 0; k < p.nk(); ++k)
    for (int x = 0; x < 3; ++x) kp[3 * k + x] = p.K[k][x];
  h2d(ctx, ctx->kpts, kp.data(), sizeof(double) * kp.size());
}

// One q of one problem, from the eigenpairs at k (wk, zk) and k+q (wq, zq):
// transitions, overlaps, contraction, scaling, Kramers-Kronig, copy-out into
// the .dat layout [i][j][q][m][n][f] of re/im (and eps_M of this q).
void chi_process_q(pmx_ctx* ctx, const Problem& p, const ChiPlan& pl, const DevCrystal& dc, int q, double off,
                   const std::vector<double>& wk, const std::vector<double>& wq, const double2* zk,
                   const double2* zq, int precision, double* re, double* im, bool device_out, double* epsm) {
  cudaStream_t st = ctx->stream;
  const int mode = pl.mode, nk = pl.nk, nq = pl.nq, neps = pl.neps, nf = pl.nf, np = pl.np;
  const int nev = pl.nev, nval = pl.nval, n = pl.n, nch = pl.nch, W = pl.W, FT = pl.FT, nft = pl.nft;
  const size_t blkvals = pl.blkvals;
  const bool pv = pl.pv;
  pmx::dev::ScaleArgs sa = pl.sa;
  const Vec3 Q = p.lat.Q[q];
  // transition list on the device (trans.cu): occupations and counts, one
  // read-back of the summary, then the list, its sort by window start and
  // the frequency-tile ranges
  pmx::dev::TransArgs ta{};
  pmx::dev::TransSummary tsum{};
  {
    KTime kt(ctx, "transitions");
    h2d(ctx, ctx->t_wk, wk.data(), sizeof(double) * (size_t)nk * nval);
    h2d(ctx, ctx->t_wq, wq.data(), sizeof(double) * (size_t)nk * nval);
    h2d(ctx, ctx->t_kw, p.KW.data(), sizeof(double) * (size_t)nk);
    const int NB = p.nband;
    CK(ctx->ncd.ensure(sizeof(int) * nk));
    CK(ctx->nvd.ensure(sizeof(int) * nk));
    CK(ctx->cbase.ensure(sizeof(int) * nk));
    CK(ctx->vbase.ensure(sizeof(int) * nk));
    CK(ctx->cidx.ensure(sizeof(int) * (size_t)nk * NB));
    CK(ctx->vidx.ensure(sizeof(int) * (size_t)nk * NB));
    CK(ctx->t_ntr.ensure(sizeof(int) * nk));
    CK(ctx->t_nblk.ensure(sizeof(int) * nk));
    CK(ctx->blkoff.ensure(sizeof(long long) * nk));
    CK(ctx->t_toff.ensure(sizeof(long long) * nk));
    CK(ctx->t_sum.ensure(sizeof(pmx::dev::TransSummary)));
    ta.wk = ctx->t_wk.as<double>();
    ta.wq = ctx->t_wq.as<double>();
    ta.kw = ctx->t_kw.as<double>();
    ta.nk = nk;
    ta.nval = nval;
    ta.nband = NB;
    ta.nh = 2 * p.npw();
    ta.soc = dc.soc;
    ta.xyz = mode == 2 ? 1 : 0;
    ta.off = off;
    ta.w0 = p.freq.empty() ? 0.0 : p.freq[0];
    ta.df = p.dfreq;
    ta.ncd = ctx->ncd.as<int>();
    ta.nvd = ctx->nvd.as<int>();
    ta.cbase = ctx->cbase.as<int>();
    ta.vbase = ctx->vbase.as<int>();
    ta.cidx = ctx->cidx.as<int>();
    ta.vidx = ctx->vidx.as<int>();
    ta.ntr = ctx->t_ntr.as<int>();
    ta.nblk = ctx->t_nblk.as<int>();
    ta.blkoff = ctx->blkoff.as<long long>();
    ta.toff = ctx->t_toff.as<long long>();
    ta.sum = ctx->t_sum.as<pmx::dev::TransSummary>();
    CK(pmx::dev::launch_transitions_count(ta, st));
    CK(cudaMemcpyAsync(&tsum, ta.sum, sizeof(tsum), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    ctx->d2h += (long long)sizeof(tsum);
    ctx->launches += 2;
    ctx->degenerate_cuts += tsum.cuts;
    ctx->occupation_ties += tsum.ties;
    const bool sort = mode == 0;
    if (sort && !pmx::dev::transitions_sortable(tsum))
      throw CudaFail("transition energies span too many frequency steps for the device sort", PMX_ERR_LIMIT);
    const size_t T0 = (size_t)std::max<long long>(tsum.T, 1);
    CK(ctx->dest.ensure(sizeof(long long) * (size_t)std::max<long long>(tsum.nblk, 1)));
    CK(ctx->dE.ensure(sizeof(double) * T0));
    CK(ctx->wgt.ensure(sizeof(double) * T0));
    CK(ctx->f0.ensure(sizeof(int) * T0));
    CK(ctx->t_rsrc.ensure(sizeof(long long) * T0));
    CK(ctx->t_rde.ensure(sizeof(double) * T0));
    CK(ctx->t_rw.ensure(sizeof(double) * T0));
    CK(ctx->t_rf0.ensure(sizeof(int) * T0));
    CK(ctx->trange.ensure(sizeof(int2) * std::max(nft, 1)));
    if (sort) CK(ctx->t_cnt.ensure(sizeof(int) * pmx::dev::transitions_sort_ints(tsum)));
    ta.rsrc = ctx->t_rsrc.as<long long>();
    ta.rde = ctx->t_rde.as<double>();
    ta.rw = ctx->t_rw.as<double>();
    ta.rf0 = ctx->t_rf0.as<int>();
    ta.dest = ctx->dest.as<long long>();
    ta.de = ctx->dE.as<double>();
    ta.wgt = ctx->wgt.as<double>();
    ta.f0 = ctx->f0.as<int>();
    ta.trange = ctx->trange.as<int2>();
    if (sort) {
      ta.cnt = ctx->t_cnt.as<int>();
      const long long nb = (long long)tsum.f0_hi - tsum.f0_lo + 1;
      ta.btot = ta.cnt + (pmx::dev::transitions_sort_ints(tsum) - (size_t)std::max<long long>(nb, 1));
    }
    CK(pmx::dev::launch_transitions_fill(ta, tsum, sort, nft, FT, nf, W, st));
    ctx->launches += tsum.T > 0 ? (sort ? 6 : 2) : 1;
  }
  const long long Tn = tsum.T;
  // per-m polarisation and SOC-current tables
  std::vector<double2> uv((size_t)neps * 9), ss((size_t)neps * 3);
  std::vector<double> qg(neps);
  for (int m = 0; m < neps; ++m) {
    const Vec3 v = Q + p.G[m];
    qg[m] = pmx::norm(v);
    double u[3][3][2];
    pmx::uvec_LT(v, u);
    std::complex<double> vs[3];
    soc_current(p, p.G[m], vs);
    for (int i = 0; i < 3; ++i) {
      std::complex<double> s(0, 0);
      for (int x = 0; x < 3; ++x) {
        uv[((size_t)m * 3 + i) * 3 + x] = make_double2(u[i][x][0], u[i][x][1]);
        s += std::conj(std::complex<double>(u[i][x][0], u[i][x][1])) * vs[x];
      }
      ss[(size_t)m * 3 + i] = make_double2(s.real(), s.imag());
    }
    if (mode == 2) {
      // epsxyz: Cartesian unit vectors, no SOC current (src/pmx_chi_copy.cpp:1203-1222)
      for (int i = 0; i < 3; ++i) {
        for (int x = 0; x < 3; ++x) uv[((size_t)m * 3 + i) * 3 + x] = make_double2(i == x ? 1.0 : 0.0, 0.0);
        ss[(size_t)m * 3 + i] = make_double2(0, 0);
      }
    }
  }
  h2d(ctx, ctx->uvec, uv.data(), sizeof(double2) * uv.size());
  h2d(ctx, ctx->ssoc, ss.data(), sizeof(double2) * ss.size());
  h2d(ctx, ctx->qgn, qg.data(), sizeof(double) * qg.size());
  const int A = 3 * neps;
  // overlaps: FP64 (overlap_kernel) for the FP64 contraction, on the tensor
  // cores (overlap_tc_kernel, split TF32, FP32 results) for the mixed one
  // automatic: tensor cores without spin-orbit coupling; with it (four spin
  // combinations per column) the FP64 kernel is faster (config 2: 3.1 vs 5.2 ms)
  const int om = ctx->overlap_mode == 1 ? (dc.soc ? 0 : 3) : ctx->overlap_mode;
  const bool tc_ovl = precision == PMX_PREC_MIXED && !pv && om != 0;
  const bool f64_ovl = !tc_ovl || om == 2;
  if (f64_ovl) CK(ctx->M.ensure(std::max<size_t>(sizeof(double2) * (size_t)Tn * A * nch, 16)));
  if (tc_ovl) {
    CK(ctx->m32.ensure(std::max<size_t>(sizeof(float2) * (size_t)Tn * A * nch, 16)));
    CK(ctx->tcerr.ensure(16));
    CK(cudaMemsetAsync(ctx->tcerr.ptr, 0, sizeof(int), st));
  }
  if (Tn > 0) {
    Timer tm(ctx, 1);
    pmx::dev::OverlapArgs oa{};
    oa.n = n;
    oa.npw = dc.npw;
    // epsxyz pairs eigenvector component p (not plane wave p) with loci[m][p]
    // over the first N_G components (src/pmx_chi_copy.cpp:1143, :1188, :1216):
    // the unresolved (soc = 0) gather on the spinor vectors does exactly that
    oa.soc = mode == 2 ? 0 : dc.soc;
    oa.nev = nev;
    oa.neps = neps;
    oa.nch = nch;
    oa.mode = mode == 2 ? 0 : mode;  // epsxyz: orbital current along x, y, z
    oa.ncd_max = tsum.ncd_max;
    oa.nvd_max = tsum.nvd_max;
    if (!pmx::dev::overlap_tiles(oa.ncd_max, oa.nvd_max, n, dc.npw, oa.cchunk, oa.vchunk) && f64_ovl)
      throw CudaFail("overlap tile does not fit in shared memory", PMX_ERR_UNSUPPORTED);
    oa.zk = zk;
    oa.zq = zq;
    oa.ncd = ctx->ncd.as<int>();
    oa.nvd = ctx->nvd.as<int>();
    oa.cbase = ctx->cbase.as<int>();
    oa.vbase = ctx->vbase.as<int>();
    oa.cidx = ctx->cidx.as<int>();
    oa.vidx = ctx->vidx.as<int>();
    oa.blkoff = ctx->blkoff.as<long long>();
    oa.dest = ctx->dest.as<long long>();
    oa.loci = ctx->loci.as<int>();
    oa.G = dc.host.G;
    oa.kpts = ctx->kpts.as<double>();
    oa.q[0] = Q.x;
    oa.q[1] = Q.y;
    oa.q[2] = Q.z;
    oa.uvec = ctx->uvec.as<double2>();
    oa.ssoc = ctx->ssoc.as<double2>();
    if (f64_ovl) {
      oa.M = ctx->M.as<double2>();
      // tile shape: cached per shape key, or timed once on a k grid of at
      // least 148 points (every candidate computes the same M; the chosen one
      // runs last)
      const std::array<int, 6> okey{n, dc.npw, oa.ncd_max, oa.nvd_max, neps, (nch << 4) | (oa.soc << 2) | oa.mode};
      auto ot = ctx->ovl_tune.find(okey);
      if (ot != ctx->ovl_tune.end()) {
        oa.cchunk = ot->second.cchunk;
        oa.vchunk = ot->second.vchunk;
      } else if (ctx->autotune && nk >= 148) {
        int cc[4], vc[4];
        const int ncand = pmx::dev::overlap_tile_candidates(oa.ncd_max, oa.nvd_max, n, dc.npw, cc, vc, 4);
        if (ncand > 1) {
          // two rounds over the candidates, the faster of each candidate's two
          // times: the first launches also warm the caches and the clocks
          pmx_ctx::OvlTune t;
          t.ms.assign(ncand, 1e30f);
          for (int round = 0; round < 2; ++round)
            for (int i = 0; i < ncand; ++i) {
              pmx::dev::OverlapArgs ob = oa;
              ob.cchunk = cc[i];
              ob.vchunk = vc[i];
              float ms = 0.f;
              CK(cudaEventRecord(ctx->ev[2], st));
              CK(pmx::dev::launch_overlap(ob, nk, st));
              CK(cudaEventRecord(ctx->ev[3], st));
              CK(cudaEventSynchronize(ctx->ev[3]));
              CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
              t.ms[i] = std::min(t.ms[i], ms);
              ctx->launches += 1;
            }
          t.cc.assign(cc, cc + ncand);
          t.vc.assign(vc, vc + ncand);
          const int best = (int)(std::min_element(t.ms.begin(), t.ms.end()) - t.ms.begin());
          t.cchunk = cc[best];
          t.vchunk = vc[best];
          oa.cchunk = t.cchunk;
          oa.vchunk = t.vchunk;
          ctx->ovl_tune[okey] = t;
        }
      }
      KTime kt(ctx, "overlap");
      CK(pmx::dev::launch_overlap(oa, nk, st));
      ctx->launches += 1;
    }
    if (tc_ovl) {
      pmx::dev::OverlapTcArgs tca{};
      tca.a = oa;
      tca.a.M = nullptr;
      tca.M32 = ctx->m32.as<float2>();
      tca.wait_ns = ctx->wait_ns;
      tca.err = ctx->tcerr.as<int>();
      tca.fault = ctx->fault;
      KTime kt(ctx, "overlap_tc");
      CK(pmx::dev::launch_overlap_tc(tca, nk, st));
      ctx->launches += 1;
    }
  }
  // contraction
  {
    Timer tm(ctx, 2);
    pmx::dev::ContractArgs ca{};
    ca.M = f64_ovl ? ctx->M.as<double2>() : nullptr;
    ca.M32 = tc_ovl ? ctx->m32.as<float2>() : nullptr;
    ca.dE = ctx->dE.as<double>();
    ca.wgt = ctx->wgt.as<double>();
    ca.f0 = ctx->f0.as<int>();
    ca.trange = ctx->trange.as<int2>();
    ca.neps = neps;
    ca.np = np;
    ca.nf = nf;
    ca.nch = nch;
    ca.window = W;
    ca.delta = p.delta;
    ca.eps = p.epsilon;
    ca.dfreq = p.dfreq;
    ca.acc = ctx->acc.as<double>();
    ca.acc_pv = pv ? ctx->accpv.as<double>() : nullptr;
    ca.pvclass = mode == 2 ? 3 : 0;
    ca.wait_ns = ctx->wait_ns;
    ca.fault = ctx->fault;
    if (precision == PMX_PREC_FP64 || pv) {
      KTime kt(ctx, "contract_f64");
      CK(pmx::dev::launch_contract_f64(ca, st));
      ctx->launches += 1;
    } else {
      int nl = 0;
      CK(ctx->mixws.ensure(std::max<size_t>(pmx::dev::mixed_workspace_bytes(ca, Tn), 16)));
      CK(ctx->stats.ensure(16));
      ca.stats = ctx->stats.as<double>();
      {
        KTime kt(ctx, "contract_mixed");
        long long mm = 0;
        const cudaError_t e = pmx::dev::launch_contract_mixed(ca, Tn, ctx->mixws.ptr, nl, st, &mm);
        if (e == cudaErrorTimeout)
          throw CudaFail("mixed contraction: a bounded device wait ran out (the CTAs returned)", PMX_ERR_TIMEOUT);
        CK(e);
        ctx->mixed_mmas += mm;
      }
      ctx->launches += nl;
      double sv[2] = {0, 0};
      int oerr = 0;
      CK(cudaMemcpyAsync(sv, ctx->stats.ptr, sizeof(sv), cudaMemcpyDeviceToHost, st));
      if (tc_ovl) CK(cudaMemcpyAsync(&oerr, ctx->tcerr.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (oerr)
        throw CudaFail("tensor-core overlaps: a bounded device wait ran out (the CTAs returned)", PMX_ERR_TIMEOUT);
      if (f64_ovl) {
        ctx->m2_err = std::max(ctx->m2_err, sv[0]);
        ctx->m2_max = std::max(ctx->m2_max, sv[1]);
      }
    }
  }
  // scaling and Kramers-Kronig
  {
    Timer tm(ctx, 3);
    sa.qgn = ctx->qgn.as<double>();
    sa.acc = ctx->acc.as<double>();
    sa.acc_pv = pv ? ctx->accpv.as<double>() : nullptr;
    sa.out = ctx->chi.as<double>();
    {
      KTime kt(ctx, "scale");
      CK(pmx::dev::launch_scale(sa, st));
    }
    ctx->launches += 1;
    if (p.kk) {
      KTime kt(ctx, "kk");
      CK(pmx::dev::launch_kk(ctx->chi.as<double>(), ctx->chi2.as<double>(), 9 * np, nf, p.dfreq, st));
      ctx->launches += 1;
    }
  }
  // copy out into [i][j][q][m][n][f]
  {
    Timer tm(ctx, 4);
    const double* res = p.kk ? ctx->chi2.as<double>() : ctx->chi.as<double>();
    const size_t row = (size_t)np * nf * sizeof(double);
    const cudaMemcpyKind kind = device_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (re) {  // NULL: eps_M only
      CK(cudaMemcpy2DAsync(re + (size_t)q * np * nf, row * nq, res, row, row, 9, kind, st));
      CK(cudaMemcpy2DAsync(im + (size_t)q * np * nf, row * nq, res + blkvals, row, row, 9, kind, st));
      if (!device_out) ctx->d2h += (long long)(2 * 9 * row);
    }
    if (epsm) {
      // eps_M of this q from the (L, L) block: [i=0][j=0] rows of res
      CK(ctx->epsm.ensure(sizeof(double2) * nf));
      CK(pmx::dev::launch_epsm(res, res + blkvals, neps, 1, nf, ctx->epsm.as<double2>(), st));
      ctx->launches += 1;
      CK(cudaMemcpyAsync(epsm + (size_t)2 * q * nf, ctx->epsm.ptr, sizeof(double2) * nf,
                         device_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
      if (!device_out) ctx->d2h += (long long)(sizeof(double2) * nf);
    }
  }
}

}  // namespace

static int run_chi(pmx_ctx* ctx, const pmx_problem* P, int sw, int precision, double* re, double* im,
                   bool device_out, double* epsm) {
  if (!P || (sw != PMX_SWITCH_EPSIJ && sw != PMX_SWITCH_EPSLL && sw != PMX_SWITCH_EPSXYZ)) return PMX_ERR_INVALID;
  if (precision != PMX_PREC_FP64 && precision != PMX_PREC_MIXED) return PMX_ERR_INVALID;
  if (epsm && sw == PMX_SWITCH_EPSXYZ) return PMX_ERR_INVALID;  // eps_M is defined on the (L, L) block
  return guarded(ctx, [&]() -> int {
    const Problem& p = P->p;
    cudaStream_t st = ctx->stream;
    for (double& t : ctx->stage_ms) t = 0;
    // re/im may both be NULL when eps_M is requested (eps_M only, no chi copy-out)
    if ((!re || !im) && !(epsm && !re && !im)) return (int)PMX_ERR_INVALID;
    DevCrystal dc;
    double off;
    std::vector<double> wk;
    {
      Timer tm(ctx, 0);
      dc = upload_crystal(ctx, P, sw == PMX_SWITCH_EPSXYZ ? 1 : 0);
      off = ref_energy(ctx, P, dc);
    }
    const ChiPlan pl = chi_plan(p, sw, dc);
    const int nk = pl.nk, nev = pl.nev, nval = pl.nval, n = pl.n;
    ctx->degenerate_cuts = 0;
    ctx->occupation_ties = 0;
    ctx->m2_err = ctx->m2_max = 0.0;
    CK(ctx->zk.ensure(std::max<size_t>(sizeof(double2) * (size_t)nk * nev * n, 16)));
    CK(ctx->zq.ensure(std::max<size_t>(sizeof(double2) * (size_t)nk * nev * n, 16)));
    {
      Timer tm(ctx, 0);
      solve_k(ctx, dc, p.K, nval, nev, ctx->zk.as<double2>(), wk);
    }
    chi_tables(ctx, p);
    chi_buffers(ctx, pl);
    for (int q = 0; q < pl.nq; ++q) {
      const Vec3 Q = p.lat.Q[q];
      std::vector<Vec3> kq(nk);
      for (int k = 0; k < nk; ++k) kq[k] = p.K[k] + Q;
      std::vector<double> wq;
      {
        Timer tm(ctx, 0);
        solve_k(ctx, dc, kq, nval, nev, ctx->zq.as<double2>(), wq);
      }
      chi_process_q(ctx, p, pl, dc, q, off, wk, wq, ctx->zk.as<double2>(), ctx->zq.as<double2>(), precision, re,
                    im, device_out, epsm);
    }
    CK(cudaStreamSynchronize(st));
    if (ctx->degenerate_cuts > 0)
      std::cerr << "WARNING: -nband " << p.nband << " cuts a degenerate set at " << ctx->degenerate_cuts
                << " k / k+q points (|E_NBAND - E_NBAND+1| < 1e-8 eV); chi then depends on the eigenvector "
                   "basis inside that set, for the reference's eigensolver as for this one"
                << std::endl;
    if (ctx->occupation_ties > 0)
      std::cerr << "WARNING: " << ctx->occupation_ties
                << " k / k+q points have a state within 1e-8 eV of the reference energy; their occupation "
                   "(E - E_ref > 0 or <= 0) and so chi are decided by rounding"
                << std::endl;
    return (int)PMX_OK;
  });
}

extern "C" int pmx_chi(pmx_ctx* ctx, const pmx_problem* P, int sw, int precision, double* re, double* im) {
  return run_chi(ctx, P, sw, precision, re, im, false, nullptr);
}

extern "C" int pmx_chi_device(pmx_ctx* ctx, const pmx_problem* P, int sw, int precision, double* re_dev,
                              double* im_dev, double* epsm_dev) {
  return run_chi(ctx, P, sw, precision, re_dev, im_dev, true, epsm_dev);
}

extern "C" int pmx_chi_epsm(pmx_ctx* ctx, const pmx_problem* P, int sw, int precision, double* re, double* im,
                            double* epsm) {
  if (P && P->p.neps > 64) return PMX_ERR_UNSUPPORTED;
  return run_chi(ctx, P, sw, precision, re, im, false, epsm);
}

extern "C" int pmx_eels(pmx_ctx* ctx, int nq, int nfreq, double dfreq, double wmin, const double* epsm,
                        double* loss, double* plasmon) {
  if (nq <= 0 || nfreq <= 0 || !(dfreq > 0) || !epsm || !loss || !plasmon) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    const size_t ne = (size_t)nq * nfreq;
    CK(ctx->epsm.ensure(sizeof(double2) * ne + sizeof(double) * (ne + 2 * (size_t)nq)));
    double2* de = ctx->epsm.as<double2>();
    double* dl = reinterpret_cast<double*>(de + ne);
    double* dp = dl + ne;
    CK(cudaMemcpyAsync(de, epsm, sizeof(double2) * ne, cudaMemcpyHostToDevice, ctx->stream));
    ctx->h2d += (long long)(sizeof(double2) * ne);
    const int fmin = std::max(0, (int)std::ceil(wmin / dfreq - 1e-9));
    {
      KTime kt(ctx, "loss");
      CK(pmx::dev::launch_loss(de, nq, nfreq, fmin, dfreq, dl, dp, ctx->stream));
    }
    ctx->launches += 1;
    CK(cudaMemcpyAsync(loss, dl, sizeof(double) * ne, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(plasmon, dp, sizeof(double) * 2 * nq, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->d2h += (long long)(sizeof(double) * (ne + 2 * (size_t)nq));
    return (int)PMX_OK;
  });
}

namespace {
std::vector<std::array<int, 9>> problem_ops(const pmx_problem* P, int flags) {
  const pmx::Problem& p = P->p;
  if ((flags & PMX_KGRID_LITTLE_GROUP_Q) && p.nq() < 1) throw std::runtime_error("the little group of q needs a q point");
  const pmx::Vec3* q = (flags & PMX_KGRID_LITTLE_GROUP_Q) ? &p.lat.Q[0] : nullptr;
  return pmx::symmetry_ops(p, (flags & PMX_KGRID_TIME_REVERSAL) != 0, q);
}
}  // namespace

extern "C" int pmx_problem_symmetry(const pmx_problem* P, int flags, int* nops, int* ops) {
  if (!P || !nops) return PMX_ERR_INVALID;
  try {
    const auto v = problem_ops(P, flags);
    *nops = (int)v.size();
    if (ops)
      for (size_t o = 0; o < v.size(); ++o)
        for (int e = 0; e < 9; ++e) ops[9 * o + e] = v[o][e];
    return PMX_OK;
  } catch (const std::exception&) {
    return PMX_ERR_INVALID;
  }
}

extern "C" int pmx_kgrid_reduce(pmx_ctx* ctx, const pmx_problem* P, const int* n, int flags, int* nirr, int* idx,
                                int* weight) {
  if (!P || !n || !nirr || n[0] <= 0 || n[1] <= 0 || n[2] <= 0 || (idx && !weight) || (!idx && weight))
    return PMX_ERR_INVALID;
  const long long N = (long long)n[0] * n[1] * n[2];
  if (N > (1LL << 28)) return PMX_ERR_LIMIT;
  return guarded(ctx, [&]() {
    const auto all = problem_ops(P, flags);
    // the operations that map this grid onto itself: M_ab != 0 only where n_a = n_b
    pmx::dev::KgridOps ops{};
    for (const auto& m : all) {
      bool ok = true;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) ok &= m[3 * a + b] == 0 || n[a] == n[b];
      if (ok && ops.n < pmx::dev::kKgridMaxOps) {
        for (int e = 0; e < 9; ++e) ops.m[ops.n][e] = m[e];
        ++ops.n;
      }
    }
    CK(ctx->kgrid.ensure(sizeof(int) * (size_t)(2 * N + 4 * N + 1)));
    int* rep = ctx->kgrid.as<int>();
    int* cnt = rep + N;
    int* didx = cnt + N;
    int* dw = didx + 3 * N;
    int* dn = dw + N;
    {
      KTime kt(ctx, "kgrid");
      CK(pmx::dev::launch_kgrid_reduce(ops, n, rep, cnt, didx, dw, dn, ctx->stream));
    }
    ctx->launches += 2;
    CK(cudaMemcpyAsync(nirr, dn, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (idx) {
      CK(cudaMemcpyAsync(idx, didx, sizeof(int) * 3 * (size_t)*nirr, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(weight, dw, sizeof(int) * (size_t)*nirr, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
    }
    ctx->d2h += (long long)sizeof(int) * (1 + (idx ? 4LL * *nirr : 0));
    return (int)PMX_OK;
  });
}

extern "C" void* pmx_ctx_stream(const pmx_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int pmx_ctx_kernel_time(const pmx_ctx* c, const char* family, double* ms, long long* launches) {
  if (!c || !family) return PMX_ERR_INVALID;
  auto it = c->ktime.find(family);
  if (ms) *ms = it == c->ktime.end() ? 0.0 : it->second.first;
  if (launches) *launches = it == c->ktime.end() ? 0 : it->second.second;
  return PMX_OK;
}

extern "C" int pmx_ctx_transfer_bytes(const pmx_ctx* c, long long* h2d_bytes, long long* d2h_bytes) {
  if (!c) return PMX_ERR_INVALID;
  if (h2d_bytes) *h2d_bytes = c->h2d;
  if (d2h_bytes) *d2h_bytes = c->d2h;
  return PMX_OK;
}

extern "C" int pmx_ctx_occupation_ties(const pmx_ctx* c) { return c ? c->occupation_ties : -1; }

extern "C" int pmx_ctx_degenerate_cuts(const pmx_ctx* c) { return c ? c->degenerate_cuts : -1; }

extern "C" int pmx_ctx_overlap_error(const pmx_ctx* c, double* max_abs2_err, double* max_abs2) {
  if (!c) return PMX_ERR_INVALID;
  if (max_abs2_err) *max_abs2_err = c->m2_err;
  if (max_abs2) *max_abs2 = c->m2_max;
  return PMX_OK;
}

extern "C" int pmx_ctx_mixed_mmas(const pmx_ctx* c, long long* mmas) {
  if (!c || !mmas) return PMX_ERR_INVALID;
  *mmas = c->mixed_mmas;
  return PMX_OK;
}

extern "C" int pmx_ctx_set_autotune(pmx_ctx* c, int on) {
  if (!c) return PMX_ERR_INVALID;
  c->autotune = on != 0;
  return PMX_OK;
}

extern "C" int pmx_ctx_set_wait_limit(pmx_ctx* c, long long ns) {
  if (!c || ns < 0) return PMX_ERR_INVALID;
  c->wait_ns = ns;
  return PMX_OK;
}

extern "C" int pmx_ctx_set_overlap_mode(pmx_ctx* c, int mode) {
  if (!c || mode < 0 || mode > 3) return PMX_ERR_INVALID;
  c->overlap_mode = mode;
  return PMX_OK;
}

extern "C" int pmx_ctx_set_fault(pmx_ctx* c, int fault) {
  if (!c || fault < 0 || fault > 4) return PMX_ERR_INVALID;
  c->fault = fault;
  return PMX_OK;
}

extern "C" int pmx_ctx_set_schedule(pmx_ctx* c, int schedule) {
  if (!c || schedule < -1) return PMX_ERR_INVALID;
  c->fixed_schedule = schedule;
  return PMX_OK;
}

extern "C" int pmx_ctx_tuning(const pmx_ctx* c, char* buf, size_t len, size_t* needed) {
  if (!c) return PMX_ERR_INVALID;
  std::ostringstream os;
  os << "{\"heev\": [";
  bool first = true;
  for (auto& kv : c->heev_choice) {
    const long long key = kv.first;
    os << (first ? "" : ", ") << "{\"n\": " << key / 2 / 1024 << ", \"nval\": " << (key / 2) % 1024
       << ", \"vectors\": " << (key % 2) << ", \"variant\": " << kv.second << ", \"trial_ms\": [";
    auto t = c->heev_trials.find(key);
    if (t != c->heev_trials.end())
      for (size_t i = 0; i < t->second.size(); ++i) os << (i ? ", " : "") << t->second[i];
    os << "]}";
    first = false;
  }
  os << "], \"overlap\": [";
  first = true;
  for (auto& kv : c->ovl_tune) {
    const auto& k = kv.first;
    const auto& t = kv.second;
    os << (first ? "" : ", ") << "{\"n\": " << k[0] << ", \"npw\": " << k[1] << ", \"ncd_max\": " << k[2]
       << ", \"nvd_max\": " << k[3] << ", \"neps\": " << k[4] << ", \"cchunk\": " << t.cchunk
       << ", \"vchunk\": " << t.vchunk << ", \"tiles\": [";
    for (size_t i = 0; i < t.cc.size(); ++i) os << (i ? ", " : "") << "[" << t.cc[i] << ", " << t.vc[i] << "]";
    os << "], \"trial_ms\": [";
    for (size_t i = 0; i < t.ms.size(); ++i) os << (i ? ", " : "") << t.ms[i];
    os << "]}";
    first = false;
  }
  os << "]}";
  const std::string s = os.str();
  if (needed) *needed = s.size() + 1;
  if (buf && len > 0) {
    const size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return PMX_OK;
}

extern "C" int pmx_eps_macroscopic(pmx_ctx* ctx, int neps, int nq, int nfreq, const double* chi_re,
                                   const double* chi_im, double* epsm) {
  if (neps < 1 || neps > 64 || nq < 0 || nfreq <= 0 || (nq > 0 && (!chi_re || !chi_im || !epsm)))
    return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    const size_t vals = (size_t)nq * neps * (neps + 1) / 2 * nfreq;
    if (vals == 0) return (int)PMX_OK;
    CK(ctx->chi.ensure(sizeof(double) * 2 * vals));
    CK(ctx->epsm.ensure(sizeof(double2) * nq * nfreq));
    CK(cudaMemcpyAsync(ctx->chi.ptr, chi_re, sizeof(double) * vals, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->chi.as<double>() + vals, chi_im, sizeof(double) * vals, cudaMemcpyHostToDevice,
                       ctx->stream));
    ctx->h2d += (long long)(2 * sizeof(double) * vals);
    CK(pmx::dev::launch_epsm(ctx->chi.as<double>(), ctx->chi.as<double>() + vals, neps, nq, nfreq,
                             ctx->epsm.as<double2>(), ctx->stream));
    ctx->launches += 1;
    CK(cudaMemcpyAsync(epsm, ctx->epsm.ptr, sizeof(double2) * nq * nfreq, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->d2h += (long long)(sizeof(double2) * nq * nfreq);
    return (int)PMX_OK;
  });
}

extern "C" int pmx_kk(pmx_ctx* ctx, int nrows, int nfreq, double dfreq, double* re, double* im) {
  if (nrows < 0 || nfreq <= 0 || (nrows > 0 && (!re || !im))) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    const size_t blk = (size_t)nrows * nfreq;
    if (blk == 0) return (int)PMX_OK;
    CK(ctx->chi.ensure(sizeof(double) * 2 * blk));
    CK(ctx->chi2.ensure(sizeof(double) * 2 * blk));
    CK(cudaMemcpyAsync(ctx->chi.ptr, re, sizeof(double) * blk, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->chi.as<double>() + blk, im, sizeof(double) * blk, cudaMemcpyHostToDevice, ctx->stream));
    CK(pmx::dev::launch_kk(ctx->chi.as<double>(), ctx->chi2.as<double>(), nrows, nfreq, dfreq, ctx->stream));
    ctx->launches += 1;
    CK(cudaMemcpyAsync(re, ctx->chi2.ptr, sizeof(double) * blk, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(im, ctx->chi2.as<double>() + blk, sizeof(double) * blk, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return (int)PMX_OK;
  });
}

// ======================================================================= adjoint
// Parameters of a problem, in this order: vg[atom][shell] (Ry, the -vg
// values after the g2 keys), then lambda_S (the -uniform_us_so_val value
// when -use_uniform_us_so is set, else one value per -us_so key, keys
// ascending), then one lambda_A per -ua_so key (ascending; -ua_so_val_g0 is
// key 0). H(k) is affine in all of them (src/pmx_epm.cpp:56-203).
namespace {

bool has_soc_params(const pmx_problem* P) {
  const pmx::Material& m = P->p.mat;
  return m.use_uniform_us || !m.Us.empty() || !m.Ua.empty();
}

std::vector<double> param_vector(const Problem& p) {
  std::vector<double> v;
  for (int a = 0; a < p.natom; ++a)
    for (int s = 0; s < p.mat.NV; ++s) v.push_back(p.mat.vg[a][s]);
  if (p.mat.use_uniform_us)
    v.push_back(p.mat.uniform_us);
  else
    for (auto& kv : p.mat.Us) v.push_back(kv.second);
  for (auto& kv : p.mat.Ua) v.push_back(kv.second);
  return v;
}

// Index (in ascending key order) of the map entry get_soc_form_factor
// (src/pmx_epm.cpp:22-50) returns for q2, or -1 when it returns 0.
int soc_key_index(const std::map<double, double>& m, double q2) {
  const double tol = 1e-2;
  if (std::abs(q2) < tol) {
    int i = 0;
    for (auto& kv : m) {
      if (kv.first == 0.0) return i;
      ++i;
    }
    return -1;
  }
  int best_i = -1, i = 0;
  double best = std::numeric_limits<double>::max();
  for (auto& kv : m) {
    const double d = std::abs(q2 - kv.first);
    if (d < best) {
      best = d;
      best_i = i;
    }
    ++i;
  }
  return best < tol ? best_i : -1;
}

// Parameter gradient from the hkl-difference accumulators: SV[d] = sum over
// ordered pairs (i != j) with hkl_i - hkl_j = d of the spin trace of
// conj(dL/dH), SSO[d'] = the same contracted with i (k+G_j)x(k+G_i).sigma,
// d' = hkl_j - hkl_i. dL/dp = Re sum_d SV[d] dV(d)/dp + Re sum_d SSO[d] dVSO(d)/dp.
void tables_to_grad(const Problem& p, const std::vector<double2>& SV, const std::vector<double2>& SSO,
                    bool soc, double* grad) {
  const int side = 4 * p.imax + 1, off = 2 * p.imax;
  const pmx::Material& mat = p.mat;
  const int nvg = p.natom * mat.NV;
  const int nls = mat.use_uniform_us ? 1 : (int)mat.Us.size();
  std::vector<double> g(nvg + nls + mat.Ua.size(), 0.0);
  const Vec3 b1 = p.lat.reciprocal[0], b2 = p.lat.reciprocal[1];
  const Vec3 b3 = p.lat.dim == 3 ? p.lat.reciprocal[2] : Vec3{0, 0, 0};
  for (int h = -off; h <= off; ++h)
    for (int k = -off; k <= off; ++k)
      for (int l = -off; l <= off; ++l) {
        if (p.lat.dim == 2 && l != 0) continue;
        if (!h && !k && !l) continue;
        const size_t idx = ((size_t)(h + off) * side + (k + off)) * side + (l + off);
        const Vec3 dG = (double(h) * b1 + double(k) * b2) + double(l) * b3;
        const double g2 = pmx::sqnorm(dG);
        const std::complex<double> sv(SV[idx].x, SV[idx].y);
        if (sv != 0.0 && g2 < mat.g2max) {
          int shell = -1;
          for (int s = 0; s < mat.NV; ++s)
            if (std::abs(mat.g2[s] - g2) < 1e-2) {
              shell = s;
              break;
            }
          if (shell >= 0 && p.natom > 0)
            for (int a = 0; a < p.natom; ++a) {
              const double ph = (-2.0 * pmx::kPi) * pmx::dot(dG, p.lat.atomic[a]);
              const std::complex<double> c(std::cos(ph), std::sin(ph));
              g[a * mat.NV + shell] += (sv * c).real() * pmx::kRy2eV / double(p.natom);
            }
        }
        if (!soc) continue;
        const std::complex<double> so(SSO[idx].x, SSO[idx].y);
        if (so == 0.0 || p.natom <= 0) continue;
        double cs = 0, sn = 0;
        for (const Vec3& t : p.lat.atomic) {
          cs += std::cos(2.0 * pmx::kPi * pmx::dot(dG, t));
          sn += std::sin(2.0 * pmx::kPi * pmx::dot(dG, t));
        }
        cs /= p.natom;
        sn /= p.natom;
        const int ils = mat.use_uniform_us ? 0 : soc_key_index(mat.Us, g2);
        if (ils >= 0) g[nvg + ils] += (so * (pmx::kRy2eV * cs)).real();
        const int ila = soc_key_index(mat.Ua, g2);
        if (ila >= 0) g[nvg + nls + ila] += (so * std::complex<double>(0.0, pmx::kRy2eV * sn)).real();
      }
  std::copy(g.begin(), g.end(), grad);
}

// Accumulates X Z^H of a batch of items into the pair accumulators.
void hgrad_items(pmx_ctx* c, const DevCrystal& dc, const double2* X, long long xs, const double2* Z, long long zs,
                 const std::vector<Vec3>& ks, int ns) {
  const int nb = (int)ks.size();
  if (nb == 0) return;
  std::vector<double> kp(3 * (size_t)nb);
  for (int b = 0; b < nb; ++b)
    for (int x = 0; x < 3; ++x) kp[3 * b + x] = ks[b][x];
  h2d(c, c->a_kp, kp.data(), sizeof(double) * kp.size());
  KTime kt(c, "adj_hgrad");
  CK(pmx::dev::launch_hgrad(X, xs, Z, zs, c->a_kp.as<double>(), nb, dc.n, dc.npw, dc.soc, ns, c->a_R.as<double2>(),
                            c->stream));
  c->launches += 1;
  // the k table is reused by the next call: keep the launches ordered
  CK(cudaStreamSynchronize(c->stream));
}

void adj_begin(pmx_ctx* c, const pmx_problem* P, const DevCrystal& dc) {
  const size_t pl = (size_t)dc.npw * dc.npw * (dc.soc ? 16 : 1);
  CK(c->a_R.ensure(sizeof(double2) * std::max<size_t>(pl, 1)));
  CK(cudaMemsetAsync(c->a_R.ptr, 0, sizeof(double2) * pl, c->stream));
  const int side = 4 * P->p.imax + 1;
  const size_t n3 = (size_t)side * side * side;
  CK(c->a_SV.ensure(sizeof(double2) * n3));
  CK(c->a_SSO.ensure(sizeof(double2) * n3));
  CK(cudaMemsetAsync(c->a_SV.ptr, 0, sizeof(double2) * n3, c->stream));
  CK(cudaMemsetAsync(c->a_SSO.ptr, 0, sizeof(double2) * n3, c->stream));
}

void adj_finish(pmx_ctx* c, const pmx_problem* P, const DevCrystal& dc, double* grad) {
  const int side = 4 * P->p.imax + 1;
  const size_t n3 = (size_t)side * side * side;
  {
    KTime kt(c, "adj_hscatter");
    CK(pmx::dev::launch_hscatter(c->a_R.as<double2>(), dc.npw, dc.soc, c->hkl.as<int>(), c->g.as<double>(),
                                 P->p.imax, c->a_SV.as<double2>(), c->a_SSO.as<double2>(), c->stream));
  }
  c->launches += 1;
  std::vector<double2> SV(n3), SSO(n3);
  CK(cudaMemcpyAsync(SV.data(), c->a_SV.ptr, sizeof(double2) * n3, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(SSO.data(), c->a_SSO.ptr, sizeof(double2) * n3, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->d2h += (long long)(2 * sizeof(double2) * n3);
  tables_to_grad(P->p, SV, SSO, dc.soc != 0, grad);
}

// Hellmann-Feynman term of the items' eigenvalues: lbar [nb][ns] on the host.
void hf_items(pmx_ctx* c, const DevCrystal& dc, const double2* Z, long long zs, const std::vector<double>& lbar,
              const std::vector<Vec3>& ks, int ns) {
  const int nb = (int)ks.size();
  if (nb == 0) return;
  h2d(c, c->a_lbk, lbar.data(), sizeof(double) * lbar.size());
  CK(c->a_X.ensure(sizeof(double2) * (size_t)nb * ns * dc.n));
  CK(pmx::dev::launch_hf_x(Z, zs, c->a_lbk.as<double>(), dc.n, ns, nb, c->a_X.as<double2>(), c->stream));
  c->launches += 1;
  hgrad_items(c, dc, c->a_X.as<double2>(), (long long)ns * dc.n, Z, zs, ks, ns);
}

// Gradient of the reference energy (E_{nv-1} + E_nv)/2 scaled by obar.
void ref_energy_grad(pmx_ctx* c, const pmx_problem* P, const DevCrystal& dc, double obar) {
  const Problem& p = P->p;
  const int nh = 2 * p.npw();
  if (!(p.nvalence > 0 && p.nvalence < nh) || obar == 0.0) return;
  const int ns = solved_states(p.nvalence + 1, dc.soc);
  std::vector<double> w;
  CK(c->zk.ensure(sizeof(double2) * (size_t)ns * dc.n));
  solve_k(c, dc, {p.refpoint}, ns, ns, c->zk.as<double2>(), w);
  std::vector<double> lb(ns, 0.0);
  const int s1 = dc.soc ? p.nvalence - 1 : (p.nvalence - 1) / 2, s2 = dc.soc ? p.nvalence : p.nvalence / 2;
  lb[s1] += 0.5 * obar;
  lb[s2] += 0.5 * obar;
  hf_items(c, dc, c->zk.as<double2>(), (long long)ns * dc.n, lb, {p.refpoint}, ns);
}

}  // namespace

extern "C" int pmx_problem_params(const pmx_problem* P, double* values, int* count) {
  if (!P || !count) return PMX_ERR_INVALID;
  const std::vector<double> v = param_vector(P->p);
  if (values) std::copy(v.begin(), v.end(), values);
  *count = (int)v.size();
  return PMX_OK;
}

extern "C" int pmx_problem_set_params(pmx_problem* P, const double* values, int count) {
  if (!P || (!values && count > 0)) return PMX_ERR_INVALID;
  Problem& p = P->p;
  if (count != (int)param_vector(p).size()) return PMX_ERR_INVALID;
  int i = 0;
  for (int a = 0; a < p.natom; ++a)
    for (int s = 0; s < p.mat.NV; ++s) p.mat.vg[a][s] = values[i++];
  if (p.mat.use_uniform_us)
    p.mat.uniform_us = values[i++];
  else
    for (auto& kv : p.mat.Us) kv.second = values[i++];
  for (auto& kv : p.mat.Ua) kv.second = values[i++];
  build_tables(*P);
  return PMX_OK;
}

extern "C" int pmx_band_vjp(pmx_ctx* ctx, const pmx_problem* P, const double* dE, double* grad) {
  if (!P || !grad || (!dE && P->p.nq() > 0)) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    const Problem& p = P->p;
    DevCrystal dc = upload_crystal(ctx, P, has_soc_params(P) ? 1 : 0);
    adj_begin(ctx, P, dc);
    const int nh = 2 * p.npw(), nq = p.nq();
    const int nkeep = std::min(p.nband, nh);
    double osum = 0.0;
    if (nkeep > 0 && nq > 0) {
      const int ns = solved_states(nkeep, dc.soc), n = dc.n;
      const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nq, ((size_t)1 << 30) / ((size_t)ns * n * 16)));
      CK(ctx->zq.ensure(sizeof(double2) * (size_t)chunk * ns * n));
      for (int q0 = 0; q0 < nq; q0 += chunk) {
        const int cnt = std::min(chunk, nq - q0);
        std::vector<Vec3> ks(p.lat.Q.begin() + q0, p.lat.Q.begin() + q0 + cnt);
        std::vector<double> w;
        solve_k(ctx, dc, ks, ns, ns, ctx->zq.as<double2>(), w);
        std::vector<double> lb((size_t)cnt * ns, 0.0);
        for (int q = 0; q < cnt; ++q)
          for (int s = 0; s < nkeep; ++s) {
            const double g = dE[(size_t)(q0 + q) * p.nband + s];
            lb[(size_t)q * ns + (dc.soc ? s : s / 2)] += g;
            osum += g;
          }
        hf_items(ctx, dc, ctx->zq.as<double2>(), (long long)ns * n, lb, ks, ns);
      }
    }
    ref_energy_grad(ctx, P, dc, -osum);
    adj_finish(ctx, P, dc, grad);
    return (int)PMX_OK;
  });
}

extern "C" int pmx_epsm_vjp(pmx_ctx* ctx, const pmx_problem* P, const double* chi_re, const double* chi_im,
                            const double* deps, double* grad) {
  if (!P || !grad || !deps) return PMX_ERR_INVALID;
  const Problem& p = P->p;
  if (p.neps < 1 || p.neps > 64) return PMX_ERR_INVALID;
  std::vector<double> fre, fim;
  if (!chi_re || !chi_im) {
    // forward chi_LL (FP64) first
    const size_t vals = (size_t)9 * p.nq() * (p.neps * (p.neps + 1) / 2) * std::max(p.nfreq, 0);
    fre.assign(vals, 0.0);
    fim.assign(vals, 0.0);
    const int rc = run_chi(ctx, P, PMX_SWITCH_EPSLL, PMX_PREC_FP64, fre.data(), fim.data(), false, nullptr);
    if (rc != PMX_OK) return rc;
    chi_re = fre.data();
    chi_im = fim.data();
  }
  return guarded(ctx, [&]() -> int {
    cudaStream_t st = ctx->stream;
    for (double& t : ctx->stage_ms) t = 0;
    const int nk = p.nk(), nq = p.nq(), neps = p.neps, nf = p.nfreq;
    const int np = neps * (neps + 1) / 2;
    if (!p.have_freq || nf <= 0 || !(p.dfreq > 0)) throw std::runtime_error("-nfreq and -dfreq are required");
    if (p.nband <= 0 || p.nband > 2 * p.npw()) throw std::runtime_error("-nband out of range");
    const size_t llv = (size_t)nq * np * nf;
    // eps_M -> chi_LL
    CK(ctx->a_chi.ensure(sizeof(double) * 2 * std::max<size_t>(llv, 1)));
    CK(cudaMemcpyAsync(ctx->a_chi.ptr, chi_re, sizeof(double) * llv, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->a_chi.as<double>() + llv, chi_im, sizeof(double) * llv, cudaMemcpyHostToDevice, st));
    ctx->h2d += (long long)(2 * sizeof(double) * llv);
    h2d(ctx, ctx->a_g, deps, sizeof(double) * 2 * (size_t)nq * nf);
    CK(ctx->a_gx.ensure(sizeof(double) * 2 * std::max<size_t>(llv, 1)));
    {
      KTime kt(ctx, "adj_epsm");
      CK(pmx::dev::launch_epsm_vjp(ctx->a_chi.as<double>(), ctx->a_chi.as<double>() + llv, ctx->a_g.as<double2>(),
                                   neps, nq, nf, ctx->a_gx.as<double>(), ctx->a_gx.as<double>() + llv, st));
    }
    ctx->launches += 1;
    DevCrystal dc;
    double off;
    {
      Timer tm(ctx, 0);
      dc = upload_crystal(ctx, P, has_soc_params(P) ? 1 : 0);
      off = ref_energy(ctx, P, dc);
    }
    adj_begin(ctx, P, dc);
    const int n = dc.n, nall = n, npw = dc.npw;
    const int ns = solved_states(p.nband, dc.soc);
    h2d(ctx, ctx->loci, p.loci.data(), sizeof(int) * p.loci.size());
    std::vector<int> linv((size_t)neps * npw, -1);
    for (int m = 0; m < neps; ++m)
      for (int q = 0; q < npw; ++q) {
        const int r = p.loci[(size_t)m * npw + q];
        if (r >= 0) linv[(size_t)m * npw + r] = q;
      }
    h2d(ctx, ctx->a_linv, linv.data(), sizeof(int) * linv.size());
    const double a_cm = p.lat.a * pmx::kAngstrom, bz = p.lat.bz_volume;
    const double sf_ll = 2.0 * bz * std::pow(pmx::kE, 2) / (pmx::kPi * pmx::kEV * a_cm);
    // The eigenvector adjoint needs the first nsx eigenpairs (a prefix of the
    // spectrum containing every state with a gradient, closed under
    // degeneracy) and the reduction H = Q T Q^H of each H(k) for the resolvent
    // of the rest; a block's reflectors must fit one eigensolver chunk.
    int nsx = std::min(n, ns + 8);
    const int kb = (int)std::max<size_t>(1, std::min<size_t>((size_t)nk, ((size_t)2 << 30) / ((size_t)n * n * 16)));
    (void)nall;
    CK(ctx->a_kk.ensure(sizeof(double) * 2 * (size_t)np * nf));
    CK(ctx->chi2.ensure(sizeof(double) * 2 * (size_t)np * nf));
    const double tau = 1e-8;  // eV: eigenvalue pairs closer than this are treated as degenerate

    for (int q = 0; q < nq; ++q) {
      const Vec3 Q = p.lat.Q[q];
      // upstream of this q on [2][np][nf]: KK transpose, then the scale factors
      const size_t rowv = (size_t)np * nf;
      CK(cudaMemcpyAsync(ctx->chi2.ptr, ctx->a_gx.as<double>() + (size_t)q * rowv, sizeof(double) * rowv,
                         cudaMemcpyDeviceToDevice, st));
      CK(cudaMemcpyAsync(ctx->chi2.as<double>() + rowv, ctx->a_gx.as<double>() + llv + (size_t)q * rowv,
                         sizeof(double) * rowv, cudaMemcpyDeviceToDevice, st));
      if (p.kk) {
        KTime kt(ctx, "adj_kk");
        CK(pmx::dev::launch_kk_t(ctx->chi2.as<double>(), ctx->a_kk.as<double>(), np, nf, p.dfreq, st));
        ctx->launches += 1;
      } else {
        CK(cudaMemcpyAsync(ctx->a_kk.ptr, ctx->chi2.ptr, sizeof(double) * 2 * rowv, cudaMemcpyDeviceToDevice, st));
      }
      std::vector<double> f1(np), f2(np);
      {
        std::vector<double> qg(neps);
        for (int m = 0; m < neps; ++m) qg[m] = pmx::norm(Q + p.G[m]);
        for (int m = 0, pp = 0; m < neps; ++m)
          for (int nn = 0; nn <= m; ++nn, ++pp) {
            f1[pp] = pmx::kPi * (sf_ll / (qg[m] * qg[nn]));
            f2[pp] = 2.0 * (sf_ll / (qg[m] * qg[nn]));
          }
      }
      h2d(ctx, ctx->a_f1, f1.data(), sizeof(double) * np);
      h2d(ctx, ctx->a_f2, f2.data(), sizeof(double) * np);

      for (int k0 = 0; k0 < nk; k0 += kb) {
        const int k1 = std::min(nk, k0 + kb), cnt = k1 - k0;
        std::vector<Vec3> ks(p.K.begin() + k0, p.K.begin() + k1), kqs(cnt);
        for (int i = 0; i < cnt; ++i) kqs[i] = ks[i] + Q;
        std::vector<double> wk, wq;
        int nvs = 0, nvl = 0;
        for (;;) {
          nvs = nsx;
          nvl = std::min(n, nsx + 1);
          CK(ctx->zk.ensure(sizeof(double2) * (size_t)cnt * nvs * n));
          CK(ctx->zq.ensure(sizeof(double2) * (size_t)cnt * nvs * n));
          CK(ctx->a_trik.ensure(sizeof(double) * 4 * (size_t)cnt * n));
          CK(ctx->a_triq.ensure(sizeof(double) * 4 * (size_t)cnt * n));
          {
            Timer tm(ctx, 0);
            solve_k(ctx, dc, ks, nvl, nvs, ctx->zk.as<double2>(), wk, ctx->a_trik.as<double>());
            // keep the reflectors of the k side while the k+q side is reduced
            std::swap(ctx->hbuf.ptr, ctx->a_hk.ptr);
            std::swap(ctx->hbuf.bytes, ctx->a_hk.bytes);
            solve_k(ctx, dc, kqs, nvl, nvs, ctx->zq.as<double2>(), wq, ctx->a_triq.as<double>());
          }
          // the projected prefix must not split a degenerate set
          bool split = false;
          if (nsx < n)
            for (int i = 0; i < cnt && !split; ++i)
              split = wk[(size_t)i * nvl + nsx] - wk[(size_t)i * nvl + nsx - 1] < tau ||
                      wq[(size_t)i * nvl + nsx] - wq[(size_t)i * nvl + nsx - 1] < tau;
          if (!split) break;
          nsx = std::min(n, nsx + 8);
        }
        int cuts = 0;
        const Transitions& T = build_transitions(p, dc.soc, nvl, wk, wq, off, false, cuts, k0, k1);
        std::vector<double> kp(3 * (size_t)cnt);
        for (int i = 0; i < cnt; ++i)
          for (int x = 0; x < 3; ++x) kp[3 * i + x] = ks[i][x];
        h2d(ctx, ctx->kpts, kp.data(), sizeof(double) * kp.size());
        h2d(ctx, ctx->ncd, T.ncd.data(), sizeof(int) * T.ncd.size());
        h2d(ctx, ctx->nvd, T.nvd.data(), sizeof(int) * T.nvd.size());
        h2d(ctx, ctx->cbase, T.cbase.data(), sizeof(int) * T.cbase.size());
        h2d(ctx, ctx->vbase, T.vbase.data(), sizeof(int) * T.vbase.size());
        h2d(ctx, ctx->cidx, T.cidx.data(), sizeof(int) * T.cidx.size());
        h2d(ctx, ctx->vidx, T.vidx.data(), sizeof(int) * T.vidx.size());
        h2d(ctx, ctx->blkoff, T.blkoff.data(), sizeof(long long) * T.blkoff.size());
        h2d(ctx, ctx->dest, T.dest.data(), sizeof(long long) * T.dest.size());
        h2d(ctx, ctx->dE, T.dE.data(), sizeof(double) * T.dE.size());
        h2d(ctx, ctx->wgt, T.wgt.data(), sizeof(double) * T.wgt.size());
        const int ncd_max = T.ncd.empty() ? 0 : *std::max_element(T.ncd.begin(), T.ncd.end());
        const int nvd_max = T.nvd.empty() ? 0 : *std::max_element(T.nvd.begin(), T.nvd.end());
        CK(ctx->a_zbk.ensure(sizeof(double2) * (size_t)cnt * ns * n));
        CK(ctx->a_zbq.ensure(sizeof(double2) * (size_t)cnt * ns * n));
        CK(cudaMemsetAsync(ctx->a_zbk.ptr, 0, sizeof(double2) * (size_t)cnt * ns * n, st));
        CK(cudaMemsetAsync(ctx->a_zbq.ptr, 0, sizeof(double2) * (size_t)cnt * ns * n, st));
        CK(ctx->a_lbk.ensure(sizeof(double) * (size_t)cnt * ns));
        CK(ctx->a_lbq.ensure(sizeof(double) * (size_t)cnt * ns));
        CK(cudaMemsetAsync(ctx->a_lbk.ptr, 0, sizeof(double) * (size_t)cnt * ns, st));
        CK(cudaMemsetAsync(ctx->a_lbq.ptr, 0, sizeof(double) * (size_t)cnt * ns, st));
        if (T.T > 0) {
          const int A = 3 * neps;
          CK(ctx->M.ensure(sizeof(double2) * (size_t)T.T * A));
          {
            Timer tm(ctx, 1);
            pmx::dev::OverlapArgs oa{};
            oa.n = n;
            oa.npw = npw;
            oa.soc = dc.soc;
            oa.nev = nvs;
            oa.neps = neps;
            oa.nch = 1;
            oa.mode = 1;
            oa.ncd_max = ncd_max;
            oa.nvd_max = nvd_max;
            if (!pmx::dev::overlap_tiles(ncd_max, nvd_max, n, npw, oa.cchunk, oa.vchunk))
              throw CudaFail("overlap tile does not fit in shared memory", PMX_ERR_UNSUPPORTED);
            oa.zk = ctx->zk.as<double2>();
            oa.zq = ctx->zq.as<double2>();
            oa.ncd = ctx->ncd.as<int>();
            oa.nvd = ctx->nvd.as<int>();
            oa.cbase = ctx->cbase.as<int>();
            oa.vbase = ctx->vbase.as<int>();
            oa.cidx = ctx->cidx.as<int>();
            oa.vidx = ctx->vidx.as<int>();
            oa.blkoff = ctx->blkoff.as<long long>();
            oa.dest = ctx->dest.as<long long>();
            oa.loci = ctx->loci.as<int>();
            oa.G = ctx->g.as<double>();
            oa.kpts = ctx->kpts.as<double>();
            oa.q[0] = Q.x;
            oa.q[1] = Q.y;
            oa.q[2] = Q.z;
            // the L row does not use the polarisation or SOC-current tables
            oa.uvec = nullptr;
            oa.ssoc = nullptr;
            oa.M = ctx->M.as<double2>();
            CK(ctx->uvec.ensure(sizeof(double2) * 9 * neps));
            CK(ctx->ssoc.ensure(sizeof(double2) * 3 * neps));
            CK(cudaMemsetAsync(ctx->uvec.ptr, 0, sizeof(double2) * 9 * neps, st));
            CK(cudaMemsetAsync(ctx->ssoc.ptr, 0, sizeof(double2) * 3 * neps, st));
            oa.uvec = ctx->uvec.as<double2>();
            oa.ssoc = ctx->ssoc.as<double2>();
            KTime kt(ctx, "overlap");
            CK(pmx::dev::launch_overlap(oa, cnt, st));
            ctx->launches += 1;
          }
          Timer tm(ctx, 2);
          CK(ctx->a_obar.ensure(sizeof(double2) * (size_t)T.T * np));
          CK(ctx->a_debar.ensure(sizeof(double) * (size_t)T.T));
          CK(cudaMemsetAsync(ctx->a_debar.ptr, 0, sizeof(double) * (size_t)T.T, st));
          pmx::dev::ContractVjpArgs ca{};
          ca.M = ctx->M.as<double2>();
          ca.dE = ctx->dE.as<double>();
          ca.wgt = ctx->wgt.as<double>();
          ca.T = (int)T.T;
          ca.neps = neps;
          ca.np = np;
          ca.nf = nf;
          ca.delta = p.delta;
          ca.eps = p.epsilon;
          ca.dfreq = p.dfreq;
          ca.gre = ctx->a_kk.as<double>();
          ca.gim = ctx->a_kk.as<double>() + rowv;
          ca.f1 = ctx->a_f1.as<double>();
          ca.f2 = p.kk ? nullptr : ctx->a_f2.as<double>();
          ca.obar = ctx->a_obar.as<double2>();
          ca.dEbar = ctx->a_debar.as<double>();
          {
            KTime kt(ctx, "adj_contract");
            CK(pmx::dev::launch_contract_vjp(ca, st));
          }
          CK(ctx->a_mbar.ensure(sizeof(double2) * (size_t)T.T * neps));
          {
            KTime kt(ctx, "adj_mbar");
            CK(pmx::dev::launch_mbar(ctx->M.as<double2>(), ctx->a_obar.as<double2>(), (int)T.T, neps,
                                     ctx->a_mbar.as<double2>(), st));
          }
          pmx::dev::ZbarArgs za{};
          za.nk = cnt;
          za.n = n;
          za.npw = npw;
          za.soc = dc.soc;
          za.nev = nvs;
          za.ns = ns;
          za.neps = neps;
          za.ncd_max = ncd_max;
          za.nvd_max = nvd_max;
          za.zk = ctx->zk.as<double2>();
          za.zq = ctx->zq.as<double2>();
          za.ncd = ctx->ncd.as<int>();
          za.nvd = ctx->nvd.as<int>();
          za.cbase = ctx->cbase.as<int>();
          za.vbase = ctx->vbase.as<int>();
          za.cidx = ctx->cidx.as<int>();
          za.vidx = ctx->vidx.as<int>();
          za.blkoff = ctx->blkoff.as<long long>();
          za.dest = ctx->dest.as<long long>();
          za.loci = ctx->loci.as<int>();
          za.linv = ctx->a_linv.as<int>();
          za.mbar = ctx->a_mbar.as<double2>();
          za.dEbar = ctx->a_debar.as<double>();
          za.zbar_k = ctx->a_zbk.as<double2>();
          za.zbar_q = ctx->a_zbq.as<double2>();
          za.lbar_k = ctx->a_lbk.as<double>();
          za.lbar_q = ctx->a_lbq.as<double>();
          {
            KTime kt(ctx, "adj_zbar");
            CK(pmx::dev::launch_zbar(za, st));
          }
          ctx->launches += 3;
        }
        // eigenproblem adjoint of both sides, then the pair accumulators
        Timer tm(ctx, 3);
        h2d(ctx, ctx->a_lamk, wk.data(), sizeof(double) * wk.size());
        h2d(ctx, ctx->a_lamq, wq.data(), sizeof(double) * wq.size());
        const size_t cz = (size_t)cnt * ns * nsx;
        CK(ctx->a_C.ensure(sizeof(double2) * 2 * cz));
        CK(ctx->a_X.ensure(sizeof(double2) * (size_t)cnt * ns * n));
        CK(ctx->a_work.ensure(sizeof(double) * (size_t)cnt * 8 * 5 * n));
        for (int side = 0; side < 2; ++side) {
          const double2* Z = side == 0 ? ctx->zk.as<double2>() : ctx->zq.as<double2>();
          const double2* Zb = side == 0 ? ctx->a_zbk.as<double2>() : ctx->a_zbq.as<double2>();
          const double* lam = side == 0 ? ctx->a_lamk.as<double>() : ctx->a_lamq.as<double>();
          const double* lb = side == 0 ? ctx->a_lbk.as<double>() : ctx->a_lbq.as<double>();
          double2* C = ctx->a_C.as<double2>();
          {
            KTime kt(ctx, "adj_eig");
            // X = Z_S' K (prefix part) ...
            CK(pmx::dev::launch_zgemm_batched(1, nsx, ns, n, Z, n, (long long)nvs * n, Zb, n, (long long)ns * n, C,
                                              nsx, (long long)ns * nsx, cnt, st));
            CK(pmx::dev::launch_eig_kmat(C, lam, nvl, lb, nsx, ns, cnt, tau, st));
            CK(pmx::dev::launch_zgemm_batched(0, n, ns, nsx, Z, n, (long long)nvs * n, C + cz, nsx,
                                              (long long)ns * nsx, ctx->a_X.as<double2>(), n, (long long)ns * n, cnt,
                                              st));
          }
          {
            // ... + P (lam_k - H)^-1 P zbar_k for the rest of the spectrum
            KTime kt(ctx, "adj_resolvent");
            pmx::dev::ResolventArgs ra{};
            ra.n = n;
            ra.ns = ns;
            ra.nsx = nsx;
            ra.nitems = cnt;
            ra.H = side == 0 ? ctx->a_hk.as<double2>() : ctx->hbuf.as<double2>();
            ra.tri = side == 0 ? ctx->a_trik.as<double>() : ctx->a_triq.as<double>();
            ra.lam = lam;
            ra.lam_stride = nvl;
            ra.Z = Z;
            ra.zs = (long long)nvs * n;
            ra.zbar = Zb;
            ra.Y = ctx->a_X.as<double2>();
            ra.work = ctx->a_work.as<double>();
            CK(pmx::dev::launch_resolvent(ra, st));
          }
          ctx->launches += 4;
          hgrad_items(ctx, dc, ctx->a_X.as<double2>(), (long long)ns * n, Z, (long long)nvs * n,
                      side == 0 ? ks : kqs, ns);
        }
      }
    }
    adj_finish(ctx, P, dc, grad);
    return (int)PMX_OK;
  });
}

// ======================================================================= batches
// Several crystals (problems) in merged launches: every eigensolve stage of all
// problems runs as one assemble + one eigensolver launch per size class
// (matrices sorted by dimension, classes = the eigensolver's register-slot
// templates), instead of one launch sequence per problem.
namespace {

struct DevCrystalSet {
  std::vector<DevCrystal> dc;  // dc[i].dev points into the shared device table
  pmx::dev::CrystalDev* table = nullptr;
};

DevCrystalSet upload_crystals(pmx_ctx* c, const pmx_problem* const* P, int count, int force_spinor = 0) {
  DevCrystalSet set;
  std::vector<size_t> og(count + 1, 0), ov(count + 1, 0);
  for (int i = 0; i < count; ++i) {
    og[i + 1] = og[i] + 3 * (size_t)P[i]->p.npw();
    ov[i + 1] = ov[i] + P[i]->vloc.size();
  }
  CK(c->b_g.ensure(std::max<size_t>(og[count], 2) * sizeof(double)));
  CK(c->b_hkl.ensure(std::max<size_t>(og[count], 2) * sizeof(int)));
  CK(c->b_vloc.ensure(std::max<size_t>(ov[count], 2) * sizeof(double)));
  CK(c->b_vso.ensure(std::max<size_t>(ov[count], 2) * sizeof(double)));
  CK(c->b_crystal.ensure(std::max(count, 1) * sizeof(pmx::dev::CrystalDev)));
  std::vector<double> G(og[count]);
  std::vector<int> H(og[count]);
  std::vector<pmx::dev::CrystalDev> tab(count);
  set.table = c->b_crystal.as<pmx::dev::CrystalDev>();
  set.dc.resize(count);
  for (int i = 0; i < count; ++i) {
    const Problem& p = P[i]->p;
    for (int g = 0; g < p.npw(); ++g)
      for (int x = 0; x < 3; ++x) {
        G[og[i] + 3 * g + x] = p.G[g][x];
        H[og[i] + 3 * g + x] = p.hkl[g][x];
      }
    CK(cudaMemcpyAsync(c->b_vloc.as<double>() + ov[i], P[i]->vloc.data(), sizeof(double) * P[i]->vloc.size(),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->b_vso.as<double>() + ov[i], P[i]->vso.data(), sizeof(double) * P[i]->vso.size(),
                       cudaMemcpyHostToDevice, c->stream));
    c->h2d += (long long)(2 * sizeof(double) * P[i]->vloc.size());
    pmx::dev::CrystalDev& cd = tab[i];
    cd.npw = p.npw();
    cd.soc = (P[i]->soc || force_spinor) ? 1 : 0;
    cd.imax = p.imax;
    cd.side = 4 * p.imax + 1;
    const double sc = 2.0 * pmx::kPi / p.lat.a;
    cd.kin = pmx::kKCON * (sc * sc);
    cd.G = c->b_g.as<double>() + og[i];
    cd.hkl = c->b_hkl.as<int>() + og[i];
    cd.vloc = reinterpret_cast<const double2*>(c->b_vloc.as<double>() + ov[i]);
    cd.vso = reinterpret_cast<const double2*>(c->b_vso.as<double>() + ov[i]);
    DevCrystal& d = set.dc[i];
    d.host = cd;
    d.dev = set.table + i;
    d.soc = cd.soc;
    d.npw = cd.npw;
    d.n = cd.soc ? 2 * cd.npw : cd.npw;
  }
  if (count > 0) {
    CK(cudaMemcpyAsync(c->b_g.ptr, G.data(), sizeof(double) * G.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->b_hkl.ptr, H.data(), sizeof(int) * H.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->b_crystal.ptr, tab.data(), sizeof(pmx::dev::CrystalDev) * count, cudaMemcpyHostToDevice,
                       c->stream));
    // the host staging vectors die with this function
    CK(cudaStreamSynchronize(c->stream));
    c->h2d += (long long)(G.size() * sizeof(double) + H.size() * sizeof(int) + tab.size() * sizeof(tab[0]));
  }
  return set;
}

// One eigenproblem of a merged solve.
struct SolveReq {
  int crystal;       // index into the crystal table
  int n, npw;        // matrix dimension and plane waves of that crystal
  Vec3 k;
  int nval, nvec;    // lowest eigenvalues / eigenvectors wanted
  long long z_off;   // double2 offset of the nvec eigenvectors in zbase
  double* w;         // host destination of the nval eigenvalues
};

// Register-slot class of the eigensolver template that runs a matrix of size n.
int heev_class(int n) {
  const int slots = (n + 31) / 32;
  const int cls[] = {2, 4, 6, 9, 13, 19, 26, 38};
  for (int c : cls)
    if (slots <= c) return c;
  return 1 << 20;
}

// All requests in one CUDA graph: the requests are sorted by n and cut into
// chunks of one eigensolver size class (one template instantiation) and at
// most h_budget bytes of H; the assembly + eigensolver launches of every chunk are
// captured into a graph, launched once, and the eigenvalues and status codes
// of all chunks come back in one copy each.
void solve_multi(pmx_ctx* c, const pmx::dev::CrystalDev* table, std::vector<SolveReq>& reqs, double2* zbase) {
  if (reqs.empty()) return;
  std::vector<int> order(reqs.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].n > reqs[b].n; });
  struct Chunk {
    int first, cnt, max_n, max_nval, max_npw, max_nvec;
  };
  std::vector<Chunk> chunks;
  std::vector<pmx::dev::EigItem> items(reqs.size());
  long long w = 0, hneed = 0, sneed = 0, rneed = 0;
  size_t i0 = 0;
  while (i0 < order.size()) {
    const int max_n = reqs[order[i0]].n, cls = heev_class(max_n);
    const size_t ld0 = (size_t)eig_ld(max_n, max_n, false);
    const size_t hmax = h_budget(ld0 * ld0 * sizeof(double2), false);
    size_t i1 = i0, hb = 0;
    while (i1 < order.size() && i1 - i0 < 4096 && heev_class(reqs[order[i1]].n) == cls) {
      const size_t ldi = (size_t)eig_ld(reqs[order[i1]].n, max_n, false);
      const size_t b = ldi * ldi * sizeof(double2);
      if (i1 > i0 && hb + b > hmax) break;
      hb += b;
      ++i1;
    }
    if (i1 < order.size() && heev_class(reqs[order[i1]].n) == cls) {
      // cut by the H or item limit with more of this class to come: a whole
      // number of waves of CTAs
      const int unit = pmx::dev::heev_batch_unit(max_n, reqs[order[i0]].nval);
      if ((int)(i1 - i0) >= unit) i1 = i0 + (i1 - i0) / unit * unit;
    }
    Chunk ch{(int)i0, (int)(i1 - i0), max_n, 1, 1, 0};
    long long h = 0, sc = 0, rb = 0;
    for (size_t i = i0; i < i1; ++i) {
      const SolveReq& r = reqs[order[i]];
      if (r.nval > r.n || r.nvec > r.nval) throw CudaFail("too many eigenvalues requested", PMX_ERR_INVALID);
      pmx::dev::EigItem& it = items[i];
      it = pmx::dev::EigItem{};
      it.crystal = r.crystal;
      it.n = r.n;
      it.nev = r.nvec;
      it.nval = r.nval;
      it.want_vec = r.nvec > 0 ? 1 : 0;
      for (int x = 0; x < 3; ++x) it.k[x] = r.k[x];
      it.h_off = h;   // the H workspace and the scratch are reused chunk after chunk
      it.w_off = w;   // eigenvalues of all chunks side by side
      it.z_off = r.z_off;
      it.s_off = sc;
      it.ld = eig_ld(r.n, max_n, false);
      it.r_off = rb;
      eig_hooks(c, it);
      h += (long long)it.ld * it.ld;
      rb += (long long)eig_rstride(r.n, max_n, false);
      ch.max_nvec = std::max(ch.max_nvec, r.nvec);
      w += r.nval;
      sc += (long long)pmx::dev::heev_scratch_doubles(r.n, r.nvec, max_n);
      ch.max_nval = std::max(ch.max_nval, r.nval);
      ch.max_npw = std::max(ch.max_npw, r.npw);
    }
    hneed = std::max(hneed, h);
    sneed = std::max(sneed, sc);
    rneed = std::max(rneed, rb);
    chunks.push_back(ch);
    i0 = i1;
  }
  const int nitems = (int)items.size();
  CK(c->hbuf.ensure(sizeof(double2) * (size_t)hneed));
  CK(c->wbuf.ensure(sizeof(double) * (size_t)w));
  CK(c->scratch.ensure(sizeof(double) * (size_t)sneed));
  CK(c->info.ensure(sizeof(int) * nitems));
  if (rneed) CK(c->rbuf.ensure(sizeof(double2) * (size_t)rneed));
  h2d(c, c->items, items.data(), sizeof(pmx::dev::EigItem) * nitems);
  pmx::dev::EigItem* dit = c->items.as<pmx::dev::EigItem>();
  int* dinfo = c->info.as<int>();
  // eigensolver schedule per chunk: fixed, cached, or timed now (before the
  // capture) on the first chunk of at least 148 matrices of its key; the
  // trial results are recomputed by the graph
  std::vector<int> variant(chunks.size(), 0);
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const Chunk& ch = chunks[ci];
    const bool vec = zbase != nullptr;
    const long long key = ((long long)ch.max_n * 1024 + ch.max_nval) * 2 + (vec ? 1 : 0);
    const int nvar = eig_variants(ch.max_n, ch.max_nval, false);
    auto cached = c->heev_choice.find(key);
    if (c->fixed_schedule >= 0) {
      variant[ci] = std::min(c->fixed_schedule, nvar - 1);
    } else if (cached != c->heev_choice.end()) {
      variant[ci] = cached->second;
    } else if (nvar > 1 && c->autotune && ch.cnt >= 148) {
      std::vector<float> ms(nvar, 0.f);
      for (int v = 0; v < nvar; ++v) {
        CK(pmx::dev::launch_assemble(table, dit + ch.first, ch.cnt, ch.max_npw, c->hbuf.as<double2>(), c->stream));
        CK(cudaEventRecord(c->ev[2], c->stream));
        CK(eig_launch(c, dit + ch.first, ch.cnt, ch.max_n, ch.max_nval, zbase ? ch.max_nvec : 0,
                      c->hbuf.as<double2>(), c->wbuf.as<double>(), zbase ? zbase : c->hbuf.as<double2>(),
                      c->scratch.as<double>(), dinfo + ch.first, v));
        CK(cudaEventRecord(c->ev[3], c->stream));
        CK(cudaEventSynchronize(c->ev[3]));
        CK(cudaEventElapsedTime(&ms[v], c->ev[2], c->ev[3]));
        c->launches += 2;
      }
      variant[ci] = (int)(std::min_element(ms.begin(), ms.end()) - ms.begin());
      c->heev_choice[key] = variant[ci];
      c->heev_trials[key] = ms;
    }
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
  cudaError_t cap = cudaSuccess;
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const Chunk& ch = chunks[ci];
    cap = pmx::dev::launch_assemble(table, dit + ch.first, ch.cnt, ch.max_npw, c->hbuf.as<double2>(), c->stream);
    if (cap != cudaSuccess) break;
    cap = eig_launch(c, dit + ch.first, ch.cnt, ch.max_n, ch.max_nval, zbase ? ch.max_nvec : 0,
                     c->hbuf.as<double2>(), c->wbuf.as<double>(), zbase ? zbase : c->hbuf.as<double2>(),
                     c->scratch.as<double>(), dinfo + ch.first, variant[ci]);
    if (cap != cudaSuccess) break;
  }
  const cudaError_t end = cudaStreamEndCapture(c->stream, &graph);
  CK(cap);
  CK(end);
  cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
  if (inst != cudaSuccess) {
    cudaGraphDestroy(graph);
    CK(inst);
  }
  {
    KTime kt(c, "solve_graph");
    const cudaError_t e = cudaGraphLaunch(exec, c->stream);
    if (e != cudaSuccess) {
      cudaGraphExecDestroy(exec);
      cudaGraphDestroy(graph);
      CK(e);
    }
  }
  c->launches += 2 * (long long)chunks.size();
  std::vector<int> info(nitems);
  std::vector<double> wv((size_t)w);
  CK(cudaMemcpyAsync(info.data(), dinfo, sizeof(int) * nitems, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(wv.data(), c->wbuf.ptr, sizeof(double) * wv.size(), cudaMemcpyDeviceToHost, c->stream));
  const cudaError_t sy = cudaStreamSynchronize(c->stream);
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  CK(sy);
  c->d2h += (long long)(sizeof(int) * nitems + sizeof(double) * wv.size());
  for (int i = 0; i < nitems; ++i) {
    if (info[i] != 0)
      throw CudaFail("eigensolver failed (status " + std::to_string(info[i]) + ")", eig_status_error(info[i]));
    const SolveReq& r = reqs[order[i]];
    std::copy(wv.begin() + items[i].w_off, wv.begin() + items[i].w_off + r.nval, r.w);
  }
}

// Reference energies of every problem in one merged solve (setRefEnergy,
// src/pmx_epm.cpp:393-428).
std::vector<double> ref_energies(pmx_ctx* c, const pmx_problem* const* P, int count, const DevCrystalSet& set) {
  std::vector<double> off(count, 0.0);
  std::vector<std::vector<double>> w(count);
  std::vector<SolveReq> reqs;
  for (int i = 0; i < count; ++i) {
    const Problem& p = P[i]->p;
    const int nh = 2 * p.npw();
    if (!(p.nvalence > 0 && p.nvalence < nh)) {
      std::cout << "WARNING::setRefEnergy:: nvalence is out of bounds for eigenvalues. Setting offset to 0."
                << std::endl;
      continue;
    }
    const DevCrystal& d = set.dc[i];
    const int nev = solved_states(p.nvalence + 1, d.soc);
    w[i].assign(nev, 0.0);
    reqs.push_back({i, d.n, d.npw, p.refpoint, nev, 0, 0, w[i].data()});
  }
  solve_multi(c, set.table, reqs, nullptr);
  for (int i = 0; i < count; ++i) {
    if (w[i].empty()) continue;
    const Problem& p = P[i]->p;
    const int soc = set.dc[i].soc, nev = (int)w[i].size();
    off[i] = (spinor_eig(w[i], nev, 0, p.nvalence - 1, soc) + spinor_eig(w[i], nev, 0, p.nvalence, soc)) / 2.0;
  }
  return off;
}

}  // namespace

extern "C" int pmx_band_batch(pmx_ctx* ctx, int count, const pmx_problem* const* problems, double* const* eband) {
  if (count < 0 || (count > 0 && (!problems || !eband))) return PMX_ERR_INVALID;
  for (int i = 0; i < count; ++i)
    if (!problems[i] || (!eband[i] && problems[i]->p.nq() > 0)) return PMX_ERR_INVALID;
  return guarded(ctx, [&]() {
    for (double& t : ctx->stage_ms) t = 0;
    Timer tm(ctx, 0);
    const DevCrystalSet set = upload_crystals(ctx, problems, count);
    const std::vector<double> off = ref_energies(ctx, problems, count, set);
    std::vector<std::vector<double>> w(count);
    std::vector<SolveReq> reqs;
    for (int i = 0; i < count; ++i) {
      const Problem& p = problems[i]->p;
      const DevCrystal& d = set.dc[i];
      const int nkeep = std::min(p.nband, 2 * p.npw());
      if (nkeep <= 0) continue;
      const int nev = solved_states(nkeep, d.soc);
      w[i].assign((size_t)p.nq() * nev, 0.0);
      for (int q = 0; q < p.nq(); ++q)
        reqs.push_back({i, d.n, d.npw, p.lat.Q[q], nev, 0, 0, w[i].data() + (size_t)q * nev});
    }
    solve_multi(ctx, set.table, reqs, nullptr);
    for (int i = 0; i < count; ++i) {
      const Problem& p = problems[i]->p;
      const int nh = 2 * p.npw(), nkeep = std::min(p.nband, nh);
      if (nkeep <= 0) {
        std::fill(eband[i], eband[i] + (size_t)p.nq() * std::max(p.nband, 0), 0.0);
        continue;
      }
      const int nev = solved_states(nkeep, set.dc[i].soc);
      for (int q = 0; q < p.nq(); ++q)
        for (int b = 0; b < p.nband; ++b)
          eband[i][(size_t)q * p.nband + b] = b < nh ? spinor_eig(w[i], nev, q, b, set.dc[i].soc) - off[i] : 0.0;
    }
    return (int)PMX_OK;
  });
}

extern "C" int pmx_chi_batch(pmx_ctx* ctx, int count, const pmx_problem* const* problems, int sw, int precision,
                             double* const* re, double* const* im, double* const* epsm) {
  if (count < 0 || (count > 0 && !problems)) return PMX_ERR_INVALID;
  if (sw != PMX_SWITCH_EPSIJ && sw != PMX_SWITCH_EPSLL && sw != PMX_SWITCH_EPSXYZ) return PMX_ERR_INVALID;
  if (precision != PMX_PREC_FP64 && precision != PMX_PREC_MIXED) return PMX_ERR_INVALID;
  if (epsm && sw == PMX_SWITCH_EPSXYZ) return PMX_ERR_INVALID;
  for (int i = 0; i < count; ++i) {
    const bool e = epsm && epsm[i];
    const double* r = re ? re[i] : nullptr;
    const double* m = im ? im[i] : nullptr;
    // chi to host (re and im), or eps_M only (neither, eps_M requested)
    if (!problems[i] || ((!r || !m) && !(e && !r && !m)) || (e && problems[i]->p.neps > 64)) return PMX_ERR_INVALID;
  }
  return guarded(ctx, [&]() -> int {
    for (double& t : ctx->stage_ms) t = 0;
    ctx->degenerate_cuts = 0;
    ctx->occupation_ties = 0;
    ctx->m2_err = ctx->m2_max = 0.0;
    DevCrystalSet set;
    std::vector<double> off;
    {
      Timer tm(ctx, 0);
      set = upload_crystals(ctx, problems, count, sw == PMX_SWITCH_EPSXYZ ? 1 : 0);
      off = ref_energies(ctx, problems, count, set);
    }
    std::vector<ChiPlan> pl;
    for (int i = 0; i < count; ++i) pl.push_back(chi_plan(problems[i]->p, sw, set.dc[i]));
    // groups of problems whose eigenvectors at k and at k+q (one q) fit the budget
    const size_t budget = (size_t)16 << 30;
    int g0 = 0;
    while (g0 < count) {
      int g1 = g0;
      size_t zb = 0;
      while (g1 < count) {
        const size_t b = sizeof(double2) * (size_t)pl[g1].nk * pl[g1].nev * pl[g1].n;
        if (g1 > g0 && zb + b > budget) break;
        zb += b;
        ++g1;
      }
      std::vector<long long> zo(g1 - g0 + 1, 0);
      for (int i = g0; i < g1; ++i)
        zo[i - g0 + 1] = zo[i - g0] + (long long)pl[i].nk * pl[i].nev * pl[i].n;
      CK(ctx->zk.ensure(std::max<size_t>(sizeof(double2) * (size_t)zo.back(), 16)));
      CK(ctx->zq.ensure(std::max<size_t>(sizeof(double2) * (size_t)zo.back(), 16)));
      // k stage of every problem of the group
      std::vector<std::vector<double>> wk(count);
      {
        Timer tm(ctx, 0);
        std::vector<SolveReq> reqs;
        for (int i = g0; i < g1; ++i) {
          const Problem& p = problems[i]->p;
          const DevCrystal& d = set.dc[i];
          wk[i].assign((size_t)pl[i].nk * pl[i].nval, 0.0);
          for (int k = 0; k < pl[i].nk; ++k)
            reqs.push_back({i, d.n, d.npw, p.K[k], pl[i].nval, pl[i].nev,
                            zo[i - g0] + (long long)k * pl[i].nev * pl[i].n, wk[i].data() + (size_t)k * pl[i].nval});
        }
        solve_multi(ctx, set.table, reqs, ctx->zk.as<double2>());
      }
      int maxq = 0;
      for (int i = g0; i < g1; ++i) maxq = std::max(maxq, pl[i].nq);
      for (int q = 0; q < maxq; ++q) {
        // k+q stage of every problem that has this q, then each problem's chi
        std::vector<std::vector<double>> wq(count);
        {
          Timer tm(ctx, 0);
          std::vector<SolveReq> reqs;
          for (int i = g0; i < g1; ++i) {
            if (q >= pl[i].nq) continue;
            const Problem& p = problems[i]->p;
            const DevCrystal& d = set.dc[i];
            wq[i].assign((size_t)pl[i].nk * pl[i].nval, 0.0);
            for (int k = 0; k < pl[i].nk; ++k)
              reqs.push_back({i, d.n, d.npw, p.K[k] + p.lat.Q[q], pl[i].nval, pl[i].nev,
                              zo[i - g0] + (long long)k * pl[i].nev * pl[i].n,
                              wq[i].data() + (size_t)k * pl[i].nval});
          }
          solve_multi(ctx, set.table, reqs, ctx->zq.as<double2>());
        }
        for (int i = g0; i < g1; ++i) {
          if (q >= pl[i].nq) continue;
          const Problem& p = problems[i]->p;
          chi_tables(ctx, p);
          chi_buffers(ctx, pl[i]);
          chi_process_q(ctx, p, pl[i], set.dc[i], q, off[i], wk[i], wq[i], ctx->zk.as<double2>() + zo[i - g0],
                        ctx->zq.as<double2>() + zo[i - g0], precision, re ? re[i] : nullptr,
                        im ? im[i] : nullptr, false, epsm ? epsm[i] : nullptr);
        }
      }
      g0 = g1;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->degenerate_cuts > 0)
      std::cerr << "WARNING: the NBAND window cuts a degenerate set at " << ctx->degenerate_cuts
                << " k / k+q points of the batch (|E_NBAND - E_NBAND+1| < 1e-8 eV)" << std::endl;
    if (ctx->occupation_ties > 0)
      std::cerr << "WARNING: " << ctx->occupation_ties
                << " k / k+q points of the batch have a state within 1e-8 eV of the reference energy; "
                   "their occupation is decided by rounding" << std::endl;
    return (int)PMX_OK;
  });
}
