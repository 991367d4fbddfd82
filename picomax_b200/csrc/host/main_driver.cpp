// pmx_main: the picomax program (src/pmx.cpp:43-206, with the epsLL dispatch
// of src_bkp/pmx.cpp:206-222) running its two stages on the GPU.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <vector>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/picomax.h"
#include "pmx_host.hpp"

namespace {

std::string cpu_model() {
  std::ifstream f("/proc/cpuinfo");
  std::string line;
  while (std::getline(f, line))
    if (line.rfind("model name", 0) == 0) {
      auto p = line.find(':');
      return p == std::string::npos ? line : line.substr(p + 2);
    }
  return "unknown";
}

unsigned long meminfo(const char* key) {
  std::ifstream f("/proc/meminfo");
  std::string tok;
  while (f >> tok) {
    if (tok == key) {
      unsigned long v = 0;
      f >> v;
      return v;
    }
    f.ignore(1 << 20, '\n');
  }
  return 0;
}

int fail(pmx_ctx* ctx, int rc, const char* what) {
  std::cout << "ERROR: " << what << " failed: " << (ctx ? pmx_ctx_last_error(ctx) : "") << " (status " << rc
            << ")" << std::endl;
  return rc == PMX_ERR_NOCONV ? 3 : 1;
}

}  // namespace

extern "C" int pmx_main(int argc, const char* const* argv) {
  using clock = std::chrono::system_clock;
  const auto t_init = clock::now();
  pmx::ArgParser inp(argc, argv);
  if (inp.has("-h") || inp.has("-help")) {
    pmx::print_doc();
    return 0;
  }
  if (inp.has("-v") || inp.has("-version")) {
    pmx::print_version();
    return 0;
  }
  // B200 build flag, not a reference option: -precision fp64|mixed
  int precision = PMX_PREC_FP64;
  if (inp.has("-precision")) {
    const std::string v = inp.value("-precision");
    if (v == "mixed")
      precision = PMX_PREC_MIXED;
    else if (v != "fp64") {
      std::cout << "unknown -precision '" << v << "' (fp64 or mixed)" << std::endl;
      return 1;
    }
  }
  pmx_problem* P = nullptr;
  const auto t0 = clock::now();
  if (pmx_problem_create(argc, argv, &P) != PMX_OK) return 1;
  pmx_problem_info info;
  pmx_problem_get_info(P, &info);
  const pmx::Problem* pp = nullptr;
  (void)pp;
  // logfile redirection (src/pmx.cpp:76-82)
  std::string wdir = ".", outname = "picomax_output";
  {
    // wdir/outputfile are needed for the log path; re-read them from argv
    if (inp.has("-wdir")) wdir = inp.value("-wdir");
    else {
      char buf[4096];
      if (getcwd(buf, sizeof buf)) wdir = buf;
    }
    if (inp.has("-outputfile")) outname = inp.value("-outputfile");
  }
  int logfile = 0;
  inp.fill_int("-logfile", logfile);
  // -npz 1: the results also as ${out}.npz (reusable output; see pmx_write_npz)
  int npz = 0;
  inp.fill_int("-npz", npz);
  if (logfile) {
    const std::string lf = wdir + "/" + outname + ".log";
    std::cout << "Output is redirected to logfile, " << lf << std::endl;
    if (!std::freopen(lf.c_str(), "w", stdout)) {
      std::cout << "Logfile may have a problem?" << std::endl;
      pmx_problem_destroy(P);
      return 1;
    }
  }
  const std::time_t tt = clock::to_time_t(t_init);
  std::string gpu = "none";
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, 0) == cudaSuccess) gpu = prop.name;
  } else {
    cudaGetLastError();
  }
  std::cout << "*********************************\n"
            << "***PicoMax 0.1 progress output***\n"
            << "*********************************\n"
            << std::ctime(&tt) << "PicoMax v0.1 (B200 build)\n"
            << "  Running on " << cpu_model() << "\n"
            << "  Using " << std::thread::hardware_concurrency() << " cores\n"
            << "  GPU: " << gpu << "\n"
            << "  Total memory: " << (meminfo("MemTotal:") / 1000) << " MB\n"
            << "  Avail memory: " << (meminfo("MemFree:") / 1000) << " MB\n"
            << "  Working dir: " << wdir << "\n"
            << "  Output file: " << outname << ".dat\n"
            << "---------------------------------\n"
            << "Parameters:\n"
            << "  gcut = " << info.gcut << "\n"
            << "  nchi = " << info.neps << "\n"
            << "  nband = " << info.nband << "\n"
            << "  nfreq = " << info.nfreq << "\n"
            << "  dfreq = " << info.dfreq << "\n"
            << "  epsilon = " << info.epsilon << "\n"
            << "  precision = " << (precision == PMX_PREC_MIXED ? "mixed" : "fp64") << "\n"
            << "---------------------------------" << std::endl;
  std::cout << "Generated Q-vector\n  Total number: " << info.nq << std::endl;
  std::cout << "Generated G-vectors\n  Number of planewaves: " << info.npw << "\n  Elapsed time: "
            << std::chrono::duration<double>(clock::now() - t0).count() << " s" << std::endl;
  std::cout << "  Number of K-vectors: " << info.nk << std::endl;
  if (info.debug > 1) {
    size_t need = 0;
    pmx_problem_dump(P, nullptr, 0, &need);
    std::vector<char> buf(need);
    pmx_problem_dump(P, buf.data(), buf.size(), &need);
    std::cout << buf.data();
    std::cout.flush();
    pmx_problem_destroy(P);
    return 0;
  }
  int rc = 0;
  if (info.sw == PMX_SWITCH_NONE) {
    pmx_problem_destroy(P);
    return 0;
  }
  pmx_ctx* ctx = nullptr;
  int st = pmx_ctx_create(0, &ctx);
  if (st != PMX_OK) {
    std::cout << "ERROR: no usable CUDA device (status " << st << "); this library has no CPU path" << std::endl;
    pmx_problem_destroy(P);
    return 1;
  }
  const auto ts = clock::now();
  if (info.sw == PMX_SWITCH_BAND) {
    std::cout << "Electronic bandstructure solver" << std::endl;
    std::vector<double> eb((size_t)info.nq * std::max(info.nband, 0));
    st = pmx_band(ctx, P, eb.data());
    if (st != PMX_OK) {
      rc = fail(ctx, st, "band solve");
    } else {
      std::cout << "  Elapsed time: " << std::chrono::duration<double>(clock::now() - ts).count() << " s"
                << std::endl;
      const std::string path = wdir + "/" + outname + ".dat";
      std::ofstream f(path, std::ios::binary);
      if (!f) {
        std::cout << "ERROR: cannot write " << path << std::endl;
        rc = 1;
      } else {
        f.write(reinterpret_cast<const char*>(eb.data()), eb.size() * sizeof(double));
      }
      if (npz && rc == 0) {
        std::vector<double> qp((size_t)info.nq * 3);
        pmx_problem_qpoints(P, qp.data());
        const char* names[2] = {"eband", "qpoints"};
        const double* data[2] = {eb.data(), qp.data()};
        const int nd[2] = {2, 2};
        const long long shp[4] = {info.nq, std::max(info.nband, 0), info.nq, 3};
        const std::string zp = wdir + "/" + outname + ".npz";
        if (pmx_write_npz(zp.c_str(), 2, names, data, nd, shp) != PMX_OK) {
          std::cout << "ERROR: cannot write " << zp << std::endl;
          rc = 1;
        }
      }
    }
  } else {
    std::cout << "Susceptibility tensor matrix solver" << std::endl;
    std::vector<double> re(info.chi_values), im(info.chi_values);
    st = pmx_chi(ctx, P, info.sw, precision, re.data(), im.data());
    if (st != PMX_OK) {
      rc = fail(ctx, st, "susceptibility");
    } else {
      double ms[5];
      pmx_ctx_stage_times(ctx, ms);
      std::cout << "  eigensolves " << ms[0] / 1e3 << " s, overlaps " << ms[1] / 1e3 << " s, contraction "
                << ms[2] / 1e3 << " s, scaling+KK " << ms[3] / 1e3 << " s (device time)" << std::endl;
      const std::string path = wdir + "/" + outname + ".dat";
      std::ofstream f(path, std::ios::binary);
      if (!f) {
        std::cout << "ERROR: cannot write " << path << std::endl;
        rc = 1;
      } else {
        f.write(reinterpret_cast<const char*>(re.data()), re.size() * sizeof(double));
        f.write(reinterpret_cast<const char*>(im.data()), im.size() * sizeof(double));
        f.close();
        if (pmx_problem_write_gpt(P) != PMX_OK) rc = 1;
      }
      if (npz && rc == 0) {
        // the .dat blocks as [3][3][nq][pairs][nfreq] with their (m, n <= m)
        // pairs, the frequencies, q vectors and local-field G vectors
        const long long npair = (long long)info.neps * (info.neps + 1) / 2;
        std::vector<double> pairs((size_t)npair * 2), freq(std::max(info.nfreq, 0)), qp((size_t)info.nq * 3),
            G((size_t)info.npw * 3), gl((size_t)info.neps * 3);
        for (long long m = 0, k = 0; m < info.neps; ++m)
          for (long long n = 0; n <= m; ++n, ++k) {
            pairs[2 * k] = (double)m;
            pairs[2 * k + 1] = (double)n;
          }
        for (int f2 = 0; f2 < info.nfreq; ++f2) freq[f2] = info.dfreq * f2;
        pmx_problem_qpoints(P, qp.data());
        pmx_problem_gvectors(P, G.data(), nullptr);
        std::copy(G.begin(), G.begin() + gl.size(), gl.begin());
        const bool blocks = 9LL * info.nq * npair * info.nfreq == info.chi_values;
        const char* names[7] = {"ReXij", "ImXij", "pairs", "freq", "qvec", "gvec", nullptr};
        const double* data[6] = {re.data(), im.data(), pairs.data(), freq.data(), qp.data(), gl.data()};
        const int r = blocks ? 5 : 1;
        const int nd[6] = {r, r, 2, 1, 2, 2};
        std::vector<long long> shp;
        for (int a = 0; a < 2; ++a) {
          if (blocks)
            shp.insert(shp.end(), {3, 3, info.nq, npair, info.nfreq});
          else
            shp.push_back(info.chi_values);
        }
        shp.insert(shp.end(), {npair, 2, info.nfreq, info.nq, 3, info.neps, 3});
        const std::string zp = wdir + "/" + outname + ".npz";
        if (pmx_write_npz(zp.c_str(), 6, names, data, nd, shp.data()) != PMX_OK) {
          std::cout << "ERROR: cannot write " << zp << std::endl;
          rc = 1;
        }
      }
      std::cout << "  Elapsed time: " << std::chrono::duration<double>(clock::now() - ts).count() << " s"
                << std::endl;
    }
  }
  pmx_ctx_destroy(ctx);
  pmx_problem_destroy(P);
  return rc;
}
