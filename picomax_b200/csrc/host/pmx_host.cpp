// Host-side problem builder for the picomax drop-in. See pmx_host.hpp.
#include "pmx_host.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <complex>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <numeric>
#include <set>
#include <sstream>
#include <stdexcept>
#include <tuple>
#include <unordered_map>

namespace pmx {

double norm(const Vec3& a) { return std::sqrt(sqnorm(a)); }

// ---------------------------------------------------------------- argv grammar
ArgParser::ArgParser(int argc, const char* const* argv) {
  for (int i = 1; i < argc; ++i) tok_.emplace_back(argv[i]);
}

bool ArgParser::has(const std::string& opt) const {
  return std::find(tok_.begin(), tok_.end(), opt) != tok_.end();
}

const std::string& ArgParser::value(const std::string& opt) const {
  static const std::string empty;
  auto it = std::find(tok_.begin(), tok_.end(), opt);
  if (it != tok_.end() && ++it != tok_.end()) return *it;
  return empty;
}

std::vector<std::string> ArgParser::vec(const std::string& opt) const {
  // Same loop shape as inputParser::vectorOption (src/pmx.hpp:213-222): a
  // missing value yields one empty element, a trailing comma an empty tail.
  std::stringstream ss(value(opt));
  std::vector<std::string> v;
  while (ss.good()) {
    std::string s;
    std::getline(ss, s, ',');
    v.push_back(s);
  }
  return v;
}

void ArgParser::fill_int(const std::string& opt, int& v) const {
  if (has(opt)) v = std::stoi(value(opt));
}
void ArgParser::fill_double(const std::string& opt, double& v) const {
  if (has(opt)) v = std::stod(value(opt));
}

static void fail(const std::string& msg) { throw std::runtime_error(msg); }

// --------------------------------------------------------------- high symmetry
// src/pmx_basis.cpp:722-788
static Vec3 highsym_fcc(const std::string& s) {
  if (s == "G") return {0, 0, 0};
  if (s == "X") return {1, 0, 0};
  if (s == "L") return {0.5, 0.5, 0.5};
  if (s == "W") return {1, 0.5, 0};
  if (s == "U") return {1, 0.25, 0.25};
  if (s == "K") return {0.75, 0.75, 0};
  fail("unknown fcc high-symmetry point '" + s + "'");
  return {};
}
static Vec3 highsym_hex(const std::string& s, double f) {
  if (s == "G") return {0, 0, 0};
  if (s == "A") return {0, 0, 0.5 / f};
  if (s == "H") return {2.0 / 3.0, 0, 0.5 / f};
  if (s == "K") return {2.0 / 3.0, 0, 0};
  if (s == "L") return {0.5, -0.5 / std::sqrt(3.0), 0.5 / f};
  if (s == "M") return {0.5, -0.5 / std::sqrt(3.0), 0};
  fail("unknown hexagonal high-symmetry point '" + s + "'");
  return {};
}
static Vec3 highsym_hex2d(const std::string& s) {
  if (s == "G") return {0, 0, 0};
  if (s == "M") return {1.0 / 3.0, 0, 0};
  if (s == "K") return {1.0 / 3.0, 1.0 / 3.0 / std::sqrt(3.0), 0};
  if (s == "Kp") return {1.0 / 3.0, -1.0 / 3.0 / std::sqrt(3.0), 0};
  fail("unknown 2D hexagonal high-symmetry point '" + s + "'");
  return {};
}

// ------------------------------------------------------------- option process
// src/pmx_io.cpp:423-503
static void input_process(const ArgParser& inp, Problem& p) {
  inp.fill_int("-debug", p.debug);
  if (inp.has("-outputfile")) p.outputfile = inp.value("-outputfile");
  if (inp.has("-wdir"))
    p.wdir = inp.value("-wdir");
  else
    p.wdir = std::filesystem::current_path().string();
  inp.fill_int("-logfile", p.logfile);
  if (inp.has("-kpointfile")) {
    p.kpointfile = inp.value("-kpointfile");
    p.kpoint = 0;
  } else {
    inp.fill_int("-kpoint", p.kpoint);
    inp.fill_int("-kpointorder", p.lat.kpointorder);
  }
  inp.fill_int("-nband", p.nband);
  inp.fill_int("-neps", p.neps);
  inp.fill_int("-nvalence", p.nvalence);
  if (inp.has("-nfreq") && inp.has("-dfreq")) {
    p.nfreq = std::stoi(inp.value("-nfreq"));
    p.dfreq = std::stod(inp.value("-dfreq"));
    p.have_freq = true;
    p.freq.resize(std::max(p.nfreq, 0));
    for (int f = 0; f < p.nfreq; ++f) p.freq[f] = p.dfreq * f;
  }
  inp.fill_int("-kk", p.kk);
  inp.fill_double("-epsilon", p.epsilon);
  inp.fill_int("-delta", p.delta);
  if (inp.has("-refpoint")) {
    auto v = inp.vec("-refpoint");
    if (v.size() != 3) fail("check the number of refpoint!");
    for (int i = 0; i < 3; ++i) p.refpoint[i] = std::stod(v[i]);
  }
}

// src/pmx_io.cpp:108-310
static void init_crystal(const ArgParser& inp, Problem& p) {
  Crystal& lat = p.lat;
  inp.fill_int("-dim", lat.dim);
  if (inp.has("-crystal")) lat.name = inp.value("-crystal");
  if (inp.has("-a"))
    lat.a = std::stod(inp.value("-a"));
  else
    fail("lattice constant (a) is a mandatory argument!");
  inp.fill_double("-f", lat.f);
  inp.fill_double("-u", lat.u);
  const double s3 = std::sqrt(3.0);
  if (lat.name == "zb" || lat.name == "rs") {
    lat.lattice = {{0, 0.5, 0.5}, {0.5, 0, 0.5}, {0.5, 0.5, 0}};
    lat.reciprocal = {{-1, 1, 1}, {1, -1, 1}, {1, 1, -1}};
    lat.bz_volume = 4.0;
    p.natom = 2;
    if (lat.name == "zb")
      lat.atomic = {{0, 0, 0}, {0.25, 0.25, 0.25}};
    else
      lat.atomic = {{0, 0, 0}, {0.5, 0, 0}};
  } else if (lat.name == "wz" || lat.name == "te") {
    lat.lattice = {{0.5, -0.5 * s3, 0}, {0.5, 0.5 * s3, 0}, {0, 0, lat.f}};
    lat.reciprocal = {{1, -1 / s3, 0}, {1, 1 / s3, 0}, {0, 0, 1.0 / lat.f}};
    lat.bz_volume = std::abs(dot(cross(lat.reciprocal[0], lat.reciprocal[1]), lat.reciprocal[2]));
    if (lat.name == "wz") {
      p.natom = 4;
      lat.atomic = {{0.5, 0.5 / s3, 0},
                    {0.5, -0.5 / s3, 0.5 * lat.f},
                    {0.5, 0.5 / s3, lat.u * lat.f},
                    {0.5, -0.5 / s3, (0.5 + lat.u) * lat.f}};
    } else {
      p.natom = 3;
      lat.atomic = {{0, 0.5 * s3 * lat.u, -1.0 / 3.0 * lat.f},
                    {1.5 * lat.u, 0, 0},
                    {0, -0.5 * s3 * lat.u, 1.0 / 3.0 * lat.f}};
    }
  } else if (lat.name == "hex") {
    lat.dim = 2;
    lat.lattice = {{0.5 * 3, -0.5 * s3, 0}, {0.5 * 3, 0.5 * s3, 0}};
    lat.reciprocal = {{1.0 / 3.0, -s3 / 3.0, 0}, {1.0 / 3.0, s3 / 3.0, 0}};
    lat.bz_volume = std::abs(dot(lat.reciprocal[0], lat.reciprocal[1]));
    p.natom = 2;
    lat.atomic = {{0, 0, 0}, {0.5, 0, 5 * s3}};
  } else {
    // The reference leaves the lattice empty and later reads reciprocal[0]
    // out of bounds; this library reports the bad preset instead.
    fail("unknown -crystal '" + lat.name + "' (expected zb, rs, wz, te or hex)");
  }
  inp.fill_int("-gsym", lat.gsym);
  inp.fill_double("-encut", lat.encut);
  {
    const double s = lat.a / 2.0 / kPi;
    lat.gcut = std::sqrt(lat.encut * (s * s) / kKCON);
  }
  inp.fill_double("-gcut", lat.gcut);
  if (inp.has("-gammazero")) {
    auto v = inp.vec("-gammazero");
    if (v.size() != 3) fail("check the number of gammazero!");
    for (int i = 0; i < 3; ++i) lat.gammazero[i] = std::stod(v[i]);
  }
  if (inp.has("-qvec")) {
    auto v = inp.vec("-qvec");
    if (v.size() % 3 != 0) fail("check the number of qvec!");
    for (size_t i = 0; i < v.size(); i += 3)
      lat.Q.push_back({std::stod(v[i]), std::stod(v[i + 1]), std::stod(v[i + 2])});
  } else if (inp.has("-qpath") != inp.has("-qnum")) {
    fail("specify both -qpath and -qnum!");
  } else if (inp.has("-qpath") && inp.has("-qnum")) {
    for (auto& s : inp.vec("-qpath")) lat.qpath.push_back(s);
    for (auto& s : inp.vec("-qnum")) lat.qnum.push_back(std::stoi(s));
    if (lat.qpath.size() < lat.qnum.size() + 1)
      fail("-qpath needs one more point than -qnum has segments");
    Vec3 v0, v1, dv;
    for (size_t i = 0; i < lat.qnum.size(); ++i) {
      if (lat.name == "zb" || lat.name == "rs") {
        v0 = highsym_fcc(lat.qpath[i]);
        v1 = highsym_fcc(lat.qpath[i + 1]);
      } else if (lat.name == "wz" || lat.name == "te") {
        v0 = highsym_hex(lat.qpath[i], lat.f);
        v1 = highsym_hex(lat.qpath[i + 1], lat.f);
      } else {
        v0 = highsym_hex2d(lat.qpath[i]);
        v1 = highsym_hex2d(lat.qpath[i + 1]);
      }
      dv = v1 - v0;
      const int n = lat.qnum[i];
      for (int j = 0; j < n; ++j) {
        lat.Q.push_back(v0 + (double(j) / double(n)) * dv);
        if (norm(lat.Q.back()) == 0) lat.Q.back() = lat.Q.back() + lat.gammazero;
      }
    }
    lat.Q.push_back(v1);
    if (norm(lat.Q.back()) == 0) lat.Q.back() = lat.Q.back() + lat.gammazero;
  }
}

// Parses "g2:value" pairs (src/pmx_io.cpp:360-380); bad pairs are reported
// on stderr and skipped, as in the reference.
static void parse_soc_pairs(const ArgParser& inp, const std::string& opt,
                            std::map<double, double>& m) {
  for (const std::string& pair : inp.vec(opt)) {
    std::stringstream ss(pair);
    std::string g2s, vs;
    if (std::getline(ss, g2s, ':') && std::getline(ss, vs)) {
      try {
        double k = std::stod(g2s);
        double v = std::stod(vs);
        m[k] = v;
      } catch (const std::exception&) {
        std::cerr << "Invalid argument for " << opt << " pair: " << pair
                  << ". Format G^2:value expected." << std::endl;
      }
    } else {
      std::cerr << "Invalid format for " << opt << " pair: " << pair
                << ". Format G^2:value expected." << std::endl;
    }
  }
}

// src/pmx_io.cpp:315-417
static void init_mater(const ArgParser& inp, Problem& p) {
  Material& mat = p.mat;
  const double tol = 1e-2;
  if (inp.has("-vg")) {
    auto v = inp.vec("-vg");
    if (v.size() % (p.natom + 1) != 0) fail("check the number of arguments for -vg!");
    mat.NV = (int)v.size() / (p.natom + 1);
    mat.vg.assign(p.natom, std::vector<double>(mat.NV));
    for (int i = 0; i < mat.NV; ++i) {
      mat.g2.push_back(std::stod(v[i]));
      for (int j = 0; j < p.natom; ++j) mat.vg[j][i] = std::stod(v[(j + 1) * mat.NV + i]);
    }
    if (mat.NV > 0) mat.g2max = mat.g2[mat.NV - 1] + tol;
  }
  if (inp.has("-use_uniform_us_so")) {
    mat.use_uniform_us = true;
    if (inp.has("-uniform_us_so_val")) {
      try {
        mat.uniform_us = std::stod(inp.value("-uniform_us_so_val"));
      } catch (const std::exception&) {
        std::cerr << "Invalid argument for -uniform_us_so_val: Must be a number." << std::endl;
      }
    } else {
      std::cerr << "Warning: -use_uniform_us_so is set, but -uniform_us_so_val is not "
                   "provided. Defaulting to 0.0 Ry."
                << std::endl;
      mat.uniform_us = 0.0;
    }
  } else if (inp.has("-us_so")) {
    mat.use_uniform_us = false;
    parse_soc_pairs(inp, "-us_so", mat.Us);
  }
  if (inp.has("-ua_so_val_g0")) {
    try {
      mat.Ua[0.0] = std::stod(inp.value("-ua_so_val_g0"));
    } catch (const std::exception&) {
      std::cerr << "Invalid argument for -ua_so_val_g0: Must be a number." << std::endl;
    }
  }
  if (inp.has("-ua_so")) parse_soc_pairs(inp, "-ua_so", mat.Ua);
}

// --------------------------------------------------------------------- G list
// src/pmx_basis.cpp:29-132. The candidate order, the arithmetic of i1*b1+i2*b2+i3*b3
// and of the norm, and the std::sort call are those of the reference, so the
// resulting order (including inside a |G| shell) is identical.
void generate_gvectors(Problem& p) {
  const Crystal& lat = p.lat;
  const double tol = 1e-6;
  const int imax = (int)std::ceil(lat.gcut);
  const int side = 2 * imax + 1;
  const int N = lat.dim == 3 ? side * side * side : side * side;
  std::vector<Vec3> G;
  std::vector<std::array<int, 3>> H;
  G.reserve(N);
  H.reserve(N);
  if (lat.dim == 3) {
    const Vec3 b1 = lat.reciprocal[0], b2 = lat.reciprocal[1], b3 = lat.reciprocal[2];
    for (int i1 = -imax; i1 <= imax; ++i1)
      for (int i2 = -imax; i2 <= imax; ++i2)
        for (int i3 = -imax; i3 <= imax; ++i3) {
          G.push_back((double(i1) * b1 + double(i2) * b2) + double(i3) * b3);
          H.push_back({i1, i2, i3});
        }
  } else if (lat.dim == 2) {
    const Vec3 b1 = lat.reciprocal[0], b2 = lat.reciprocal[1];
    for (int i1 = -imax; i1 <= imax; ++i1)
      for (int i2 = -imax; i2 <= imax; ++i2) {
        G.push_back(double(i1) * b1 + double(i2) * b2);
        H.push_back({i1, i2, 0});
      }
  } else {
    fail("-dim must be 2 or 3");
  }
  std::vector<double> gnorm(N);
  for (int i = 0; i < N; ++i) gnorm[i] = norm(G[i]);
  std::vector<int> index(N);
  std::iota(index.begin(), index.end(), 0);
  std::sort(index.begin(), index.end(), [&](int A, int B) -> bool { return gnorm[A] < gnorm[B]; });
  std::sort(gnorm.begin(), gnorm.end(), std::less<double>());
  int npw = N;
  if (lat.gsym) {
    for (int i = 0; i < N; ++i)
      if (gnorm[i] > lat.gcut + tol) {
        npw = i;
        break;
      }
  }
  p.imax = imax;
  p.G.resize(npw);
  p.hkl.resize(npw);
  for (int i = 0; i < npw; ++i) {
    p.G[i] = G[index[i]];
    p.hkl[i] = H[index[i]];
  }
}

// src/pmx_basis.cpp:142-179. loci[m][p] = i with G_i = G_p + G_m, or -1. The
// reference searches with a 1e-10 tolerance on the difference of lattice
// vectors, which is the integer identity of their hkl.
void generate_loci(Problem& p) {
  const int npw = p.npw();
  if (p.neps > npw) fail("-neps exceeds the number of plane waves");
  if (p.neps < 1) fail("-neps must be at least 1");
  const int side = 4 * p.imax + 1;
  auto key = [&](int h, int k, int l) {
    return ((int64_t)(h + 2 * p.imax) * side + (k + 2 * p.imax)) * side + (l + 2 * p.imax);
  };
  std::unordered_map<int64_t, int> where;
  where.reserve(npw * 2);
  for (int i = 0; i < npw; ++i) where[key(p.hkl[i][0], p.hkl[i][1], p.hkl[i][2])] = i;
  p.loci.assign((size_t)p.neps * npw, -1);
  for (int q = 0; q < npw; ++q) p.loci[q] = q;
  for (int m = 1; m < p.neps; ++m) {
    for (int q = 0; q < npw; ++q) {
      const int h = p.hkl[q][0] + p.hkl[m][0];
      const int k = p.hkl[q][1] + p.hkl[m][1];
      const int l = p.hkl[q][2] + p.hkl[m][2];
      auto it = where.find(key(h, k, l));
      p.loci[(size_t)m * npw + q] = it == where.end() ? -1 : it->second;
    }
  }
}

// ------------------------------------------------------------------- k-points
// src/pmx_basis.cpp:200-245
// Reads the kpointfile format of import_kpt (src/pmx_basis.cpp:200-245):
// total count, listed count, then "kx ky kz w" per point. The reference
// leaves the points a short or malformed file does not list at k = 0 with
// weight 0 and divides by a zero total; this library rejects such files.
void import_kpoints(Problem& p) {
  std::ifstream in(p.kpointfile);
  if (!in.is_open()) fail("cannot open kpointfile '" + p.kpointfile + "'");
  int i = 0, nk0 = 0, nk = 0;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    if (i == 0) {
      if (!(std::stringstream(line) >> nk0) || nk0 <= 0) fail("kpointfile: the first line must be the total k count");
      ++i;
    } else if (i == 1) {
      if (!(std::stringstream(line) >> nk) || nk < 0) fail("kpointfile: the second line must be the listed k count");
      p.K.assign(nk, Vec3{});
      p.KW.assign(nk, 0.0);
      ++i;
    } else if (i - 2 < nk) {
      if (!(std::stringstream(line) >> p.K[i - 2].x >> p.K[i - 2].y >> p.K[i - 2].z >> p.KW[i - 2]))
        fail("kpointfile: point " + std::to_string(i - 2) + " is not 'kx ky kz w'");
      p.KW[i - 2] /= nk0;
      ++i;
    }
  }
  if (i < 2) fail("kpointfile '" + p.kpointfile + "' has no k counts");
  if (i - 2 < nk)
    fail("kpointfile '" + p.kpointfile + "' declares " + std::to_string(nk) + " points but lists " +
         std::to_string(i - 2));
}

static bool inbz_fcc(const Vec3& K) {
  const double tol = 1e-6;
  return !(std::abs(K.x) > 1.0 + tol || std::abs(K.y) > 1.0 + tol || std::abs(K.z) > 1.0 + tol ||
           std::abs(K.x) + std::abs(K.y) + std::abs(K.z) > 1.5 + tol);
}
static bool onbz_fcc(const Vec3& K) {
  const double tol = 1e-6;
  return std::abs(std::abs(K.x) - 1.0) < tol || std::abs(std::abs(K.y) - 1.0) < tol ||
         std::abs(std::abs(K.z) - 1.0) < tol ||
         std::abs(std::abs(K.x) + std::abs(K.y) + std::abs(K.z) - 1.5) < tol;
}
static bool inbz_hex(const Vec3& K, double f) {
  const double tol = 1e-6;
  return !(std::abs(K.z) > 0.5 / f + tol || std::abs(K.y) > 1.0 / std::sqrt(3.0) + tol ||
           std::abs(K.x) + std::abs(K.y) / std::sqrt(3.0) > 1.0 / std::sqrt(3.0) + tol);
}
static bool inbz_hex2(const Vec3& K) {
  const double tol = 1e-6;
  return !(std::abs(K.y) > 1.0 / std::sqrt(3.0) + tol ||
           std::abs(K.x) + std::abs(K.y) / std::sqrt(3.0) > 1.0 / std::sqrt(3.0) + tol);
}

// src/pmx_basis.cpp:604-650
static void kpt_fcc2(Problem& p) {
  const int N = p.lat.kpointorder;
  const Vec3 b1 = p.lat.reciprocal[0], b2 = p.lat.reciprocal[1], b3 = p.lat.reciprocal[2];
  const double df = 1.0 / N;
  std::vector<Vec3> K;
  std::vector<double> W;
  for (int i1 = -N; i1 <= N; ++i1)
    for (int i2 = -N; i2 <= N; ++i2)
      for (int i3 = -N; i3 <= N; ++i3)
        K.push_back(((df * i1) * b1 + (df * i2) * b2) + (df * i3) * b3);
  W.resize(K.size());
  double w0 = 0;
  for (size_t i = 0; i < K.size(); ++i) {
    W[i] = !inbz_fcc(K[i]) ? 0.0 : (onbz_fcc(K[i]) ? 0.5 : 1.0);
    w0 += W[i];
  }
  p.K.clear();
  p.KW.clear();
  for (size_t i = 0; i < K.size(); ++i)
    if (W[i] != 0) {
      p.K.push_back(K[i]);
      p.KW.push_back(W[i] / w0);
    }
}

// src/pmx_basis.cpp:413-496
static void symmetrize_xy_hex(Problem& p) {
  typedef std::tuple<double, double, double> Key;
  const double tol = 1e-9;
  auto mk = [&](double x, double y, double z) {
    return Key{std::round(x / tol) * tol, std::round(y / tol) * tol, std::round(z / tol) * tol};
  };
  std::map<Key, double> uw;
  for (size_t i = 0; i < p.K.size(); ++i) uw[mk(p.K[i].x, p.K[i].y, p.K[i].z)] += p.KW[i];
  std::map<Key, double> sw;
  std::set<Key> done;
  for (const auto& kv : uw) {
    const Key& k = kv.first;
    if (done.count(k)) continue;
    const Key ks = mk(std::get<1>(k), std::get<0>(k), std::get<2>(k));
    done.insert(k);
    done.insert(ks);
    if (k == ks) {
      sw[k] += kv.second;
    } else {
      double w2 = 0.0;
      auto it = uw.find(ks);
      if (it != uw.end()) w2 = it->second;
      const double c = kv.second + w2;
      sw[k] += c / 2.0;
      sw[ks] += c / 2.0;
    }
  }
  p.K.clear();
  p.KW.clear();
  double tot = 0;
  for (const auto& kv : sw) {
    p.K.push_back({std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first)});
    p.KW.push_back(kv.second);
    tot += kv.second;
  }
  if (tot > 0)
    for (double& w : p.KW) w /= tot;
}

// src/pmx_basis.cpp:499-546
static void kpt_hex(Problem& p) {
  const int N = p.lat.kpointorder;
  const Vec3 b1 = p.lat.reciprocal[0], b2 = p.lat.reciprocal[1], b3 = p.lat.reciprocal[2];
  const double df = 1.0 / N;
  p.K.clear();
  for (int i1 = 0; i1 < N; ++i1)
    for (int i2 = 0; i2 < N; ++i2)
      for (int i3 = 0; i3 < N; ++i3)
        p.K.push_back(((df * i1) * b1 + (df * i2) * b2) + (df * i3) * b3);
  for (auto& K : p.K) {
    if (inbz_hex(K, p.lat.f)) continue;
    bool moved = false;
    for (int s1 = -1; s1 <= 1 && !moved; ++s1)
      for (int s2 = -1; s2 <= 1 && !moved; ++s2)
        for (int s3 = -1; s3 <= 1 && !moved; ++s3) {
          if (inbz_hex(((K + double(s1) * b1) + double(s2) * b2) + double(s3) * b3, p.lat.f)) {
            K = K + ((double(s1) * b1 + double(s2) * b2) + double(s3) * b3);
            moved = true;
          }
        }
  }
  p.KW.assign(p.K.size(), 1.0 / double(p.K.size()));
  symmetrize_xy_hex(p);
}

// src/pmx_basis.cpp:551-599. The reference scans 27 entries of a 9-entry shift
// table (reading past its end); only the 9 real shifts are scanned here.
static void kpt_hex2(Problem& p) {
  const int N = p.lat.kpointorder;
  const Vec3 b1 = p.lat.reciprocal[0], b2 = p.lat.reciprocal[1];
  const double df = 1.0 / N;
  p.K.clear();
  for (int i1 = 0; i1 < N; ++i1)
    for (int i2 = 0; i2 < N; ++i2) p.K.push_back((df * i1) * b1 + (df * i2) * b2);
  for (auto& K : p.K) {
    if (inbz_hex2(K)) continue;
    bool moved = false;
    for (int s1 = -1; s1 <= 1 && !moved; ++s1)
      for (int s2 = -1; s2 <= 1 && !moved; ++s2)
        if (inbz_hex2((K + double(s1) * b1) + double(s2) * b2)) {
          K = K + (double(s1) * b1 + double(s2) * b2);
          moved = true;
        }
  }
  p.KW.assign(p.K.size(), 1.0 / double(p.K.size()));
}

void generate_kpoints_bz(Problem& p) {
  const std::string& n = p.lat.name;
  if (n == "zb" || n == "rs")
    kpt_fcc2(p);
  else if (n == "wz" || n == "te")
    kpt_hex(p);
  else if (n == "hex")
    kpt_hex2(p);
}

// src/pmx_basis.cpp:256-335 (Cohen-Chadi special points, PRB 8, 5757 (1973);
// higher orders from Phil. Mag. B 81, 551 (2001)).
void generate_kpoints_cohen_chadi(Problem& p) {
  const int N = p.lat.kpointorder;
  const int nk = int(std::pow(2.0, N - 1) * (std::pow(2.0, N) + 1.0) * (std::pow(2.0, N - 1.0) + 1.0) / 3.0);
  p.K.assign(std::max(nk, 0), Vec3{});
  p.KW.assign(std::max(nk, 0), 0.0);
  if (N == 1) {
    p.KW[0] = 0.75; p.K[0] = {0.75, 0.25, 0.25};
    p.KW[1] = 0.25; p.K[1] = {0.25, 0.25, 0.25};
  } else if (N == 2) {
    const double t[10][4] = {{0.18750, 0.875, 0.375, 0.125}, {0.09375, 0.875, 0.125, 0.125},
                             {0.09375, 0.625, 0.625, 0.125}, {0.09375, 0.625, 0.375, 0.375},
                             {0.18750, 0.625, 0.375, 0.125}, {0.09375, 0.625, 0.125, 0.125},
                             {0.03125, 0.375, 0.375, 0.375}, {0.09375, 0.375, 0.375, 0.125},
                             {0.09375, 0.375, 0.125, 0.125}, {0.03125, 0.125, 0.125, 0.125}};
    for (int k = 0; k < 10; ++k) {
      p.KW[k] = t[k][0];
      p.K[k] = {t[k][1], t[k][2], t[k][3]};
    }
  } else if (N > 2) {
    int k = 0;
    const double den = std::pow(2, N + 1);
    const double wden = 4.0 * std::pow(8.0, N - 1);
    auto put = [&](int i, int j, int l) {
      if (k >= nk) fail("Cohen-Chadi point count overflow");
      p.KW[k] = (3.0 * (1.0 - (i == j)) + 3.0 * (1.0 - (j == l)) + (i == l)) / wden;
      p.K[k] = {(2.0 * double(i) - 1) / den, (2.0 * double(j) - 1) / den, (2.0 * double(l) - 1) / den};
      ++k;
    };
    const double P1 = std::pow(2, N - 1), P0 = std::pow(2, N), P2 = std::pow(2, N - 2);
    for (int i = 1; i <= P1; i++)
      for (int j = 1; j <= i; j++)
        for (int l = 1; l <= j; l++) put(i, j, l);
    for (int i = P1 + 2; i <= P0; i += 2)
      for (int j = 1; j <= 3 * P2 - int(i * 0.5); j++)
        for (int l = 1; l <= j; l++) put(i, j, l);
    for (int i = P1 + 2; i <= 3 * P2; i += 2)
      for (int j = 3 * P2 - int(i * 0.5) + 1; j <= i; j++)
        for (int l = 1; l <= 3 * P1 + 1 - i - j; l++) put(i, j, l);
    for (int i = 3 * P2 + 2; i <= P0; i += 2)
      for (int j = 3 * P2 - int(i * 0.5) + 1; j <= 3 * P1 - i; j++)
        for (int l = 1; l <= 3 * P1 + 1 - i - j; l++) put(i, j, l);
    for (int i = P1 + 1; i <= P0 - 1; i += 2)
      for (int j = 1; j <= 3 * P2 - int((i - 1) * 0.5); j++)
        for (int l = 1; l <= j; l++) put(i, j, l);
    for (int i = P1 + 1; i <= 3 * P2 - 1; i += 2)
      for (int j = 3 * P2 - int((i - 1) * 0.5) + 1; j <= i; j++)
        for (int l = 1; l <= 3 * P1 + 1 - i - j; l++) put(i, j, l);
    for (int i = 3 * P2 + 1; i <= P0 - 1; i += 2)
      for (int j = 3 * P2 - int((i - 1) * 0.5) + 1; j <= 3 * P1 - i; j++)
        for (int l = 1; l <= 3 * P1 + 1 - i - j; l++) put(i, j, l);
  }
}

// --------------------------------------------------------------- form factors
double soc_form_factor(const std::map<double, double>& m, double q2) {
  const double tol = 1e-2;
  if (std::abs(q2) < tol) {
    auto it = m.find(0.0);
    return it != m.end() ? it->second : 0.0;
  }
  double key = 0.0, best = std::numeric_limits<double>::max();
  for (const auto& kv : m) {
    const double d = std::abs(q2 - kv.first);
    if (d < best) {
      best = d;
      key = kv.first;
    }
  }
  return best < tol ? m.at(key) : 0.0;
}

void local_potential(const Problem& p, const Vec3& dG, double& re, double& im) {
  re = im = 0;
  const Material& mat = p.mat;
  const double g2 = sqnorm(dG);
  if (!(g2 < mat.g2max)) return;
  int idx = -1;
  for (int k = 0; k < mat.NV; ++k)
    if (std::abs(mat.g2[k] - g2) < 1e-2) {
      idx = k;
      break;
    }
  if (idx < 0 || p.natom <= 0) return;
  double sr = 0, si = 0;
  for (int s = 0; s < p.natom; ++s) {
    const double ph = (-2.0 * kPi) * dot(dG, p.lat.atomic[s]);
    const double v = mat.vg[s][idx];
    sr += std::cos(ph) * v;
    si += std::sin(ph) * v;
  }
  re = sr / double(p.natom) * kRy2eV;
  im = si / double(p.natom) * kRy2eV;
}

void soc_scalar(const Problem& p, const Vec3& q, double& re, double& im) {
  const Material& mat = p.mat;
  const double q2 = sqnorm(q);
  const double ls = (mat.use_uniform_us ? mat.uniform_us : soc_form_factor(mat.Us, q2)) * kRy2eV;
  const double la = soc_form_factor(mat.Ua, q2) * kRy2eV;
  double cs = 0, sn = 0;
  if (p.natom > 0) {
    for (const Vec3& t : p.lat.atomic) {
      cs += std::cos(2.0 * kPi * dot(q, t));
      sn += std::sin(2.0 * kPi * dot(q, t));
    }
    cs /= p.natom;
    sn /= p.natom;
  }
  re = ls * cs;
  im = la * sn;
}

std::vector<std::array<int, 9>> symmetry_ops(const Problem& p, bool time_reversal, const Vec3* little_q) {
  if (p.lat.dim != 3 || p.lat.reciprocal.size() != 3)
    throw std::runtime_error("symmetry operations need a 3D crystal");
  // columns of Bm are the reciprocal basis vectors: G = Bm hkl
  double Bm[3][3], Bi[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) Bm[r][c] = p.lat.reciprocal[c][r];
  {
    const double det = Bm[0][0] * (Bm[1][1] * Bm[2][2] - Bm[1][2] * Bm[2][1]) -
                       Bm[0][1] * (Bm[1][0] * Bm[2][2] - Bm[1][2] * Bm[2][0]) +
                       Bm[0][2] * (Bm[1][0] * Bm[2][1] - Bm[1][1] * Bm[2][0]);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        const int r1 = (c + 1) % 3, r2 = (c + 2) % 3, c1 = (r + 1) % 3, c2 = (r + 2) % 3;
        Bi[r][c] = (Bm[r1][c1] * Bm[r2][c2] - Bm[r1][c2] * Bm[r2][c1]) / det;
      }
  }
  auto gvec = [&](const std::array<int, 3>& h) {
    Vec3 g;
    for (int r = 0; r < 3; ++r) g[r] = Bm[r][0] * h[0] + Bm[r][1] * h[1] + Bm[r][2] * h[2];
    return g;
  };
  // the G list (hkl) and its distinct differences
  std::set<std::array<int, 3>> gset(p.hkl.begin(), p.hkl.end());
  std::set<std::array<int, 3>> dset;
  for (const auto& a : p.hkl)
    for (const auto& b : p.hkl) dset.insert({a[0] - b[0], a[1] - b[1], a[2] - b[2]});
  std::vector<std::array<int, 3>> diffs(dset.begin(), dset.end());
  std::vector<std::complex<double>> V(diffs.size()), S(diffs.size());
  const bool soc = soc_active(p);
  double vmax = 0, smax = 0;
  for (size_t d = 0; d < diffs.size(); ++d) {
    double re, im;
    const Vec3 dg = gvec(diffs[d]);
    local_potential(p, dg, re, im);
    V[d] = {re, im};
    vmax = std::max(vmax, std::abs(V[d]));
    if (soc) {
      soc_scalar(p, (-1.0) * dg, re, im);
      S[d] = {re, im};
      smax = std::max(smax, std::abs(S[d]));
    }
  }
  std::map<std::array<int, 3>, size_t> dindex;
  for (size_t d = 0; d < diffs.size(); ++d) dindex[diffs[d]] = d;
  auto mat_apply = [](const std::array<int, 9>& M, const std::array<int, 3>& h) {
    return std::array<int, 3>{M[0] * h[0] + M[1] * h[1] + M[2] * h[2], M[3] * h[0] + M[4] * h[1] + M[5] * h[2],
                              M[6] * h[0] + M[7] * h[1] + M[8] * h[2]};
  };
  std::vector<std::array<int, 9>> ops;
  std::array<int, 9> M;
  for (int code = 0; code < 19683; ++code) {
    int c = code;
    for (int e = 0; e < 9; ++e) {
      M[e] = c % 3 - 1;
      c /= 3;
    }
    // R = Bm M Bm^-1 must be orthogonal
    double R[3][3];
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) {
        double acc = 0;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) acc += Bm[r][a] * M[3 * a + b] * Bi[b][cc];
        R[r][cc] = acc;
      }
    bool orth = true;
    for (int a = 0; a < 3 && orth; ++a)
      for (int b = 0; b < 3 && orth; ++b) {
        double acc = 0;
        for (int r = 0; r < 3; ++r) acc += R[r][a] * R[r][b];
        orth = std::abs(acc - (a == b ? 1.0 : 0.0)) < 1e-9;
      }
    if (!orth) continue;
    bool gok = true;
    for (const auto& h : p.hkl)
      if (!gset.count(mat_apply(M, h))) {
        gok = false;
        break;
      }
    if (!gok) continue;
    // translations: t = tau_j - R tau_0
    auto rot = [&](const Vec3& v) {
      Vec3 o;
      for (int r = 0; r < 3; ++r) o[r] = R[r][0] * v[0] + R[r][1] * v[1] + R[r][2] * v[2];
      return o;
    };
    bool found = false;
    const int na = std::max(1, (int)p.lat.atomic.size());
    for (int j = 0; j < na && !found; ++j) {
      const Vec3 t = p.lat.atomic.empty() ? Vec3{} : p.lat.atomic[j] - rot(p.lat.atomic[0]);
      bool ok = true;
      for (size_t d = 0; d < diffs.size() && ok; ++d) {
        const auto hr = mat_apply(M, diffs[d]);
        const auto it = dindex.find(hr);
        if (it == dindex.end()) {
          ok = false;
          break;
        }
        const double ph = -2.0 * kPi * dot(gvec(hr), t);
        const std::complex<double> e(std::cos(ph), std::sin(ph));
        ok = std::abs(V[it->second] - V[d] * e) <= 1e-9 * std::max(vmax, 1e-300) &&
             (!soc || std::abs(S[it->second] - S[d] * e) <= 1e-9 * std::max(smax, 1e-300));
      }
      found = ok;
    }
    if (!found) continue;
    ops.push_back(M);
  }
  if (time_reversal) {
    std::set<std::array<int, 9>> all(ops.begin(), ops.end());
    for (const auto& m : std::vector<std::array<int, 9>>(ops)) {
      std::array<int, 9> n;
      for (int e = 0; e < 9; ++e) n[e] = -m[e];
      all.insert(n);
    }
    ops.assign(all.begin(), all.end());
  }
  if (little_q) {  // keep the operations with M kq = kq (kq: reduced coordinates of q)
    double kq[3];
    for (int r = 0; r < 3; ++r) kq[r] = Bi[r][0] * little_q->x + Bi[r][1] * little_q->y + Bi[r][2] * little_q->z;
    std::vector<std::array<int, 9>> keep;
    for (const auto& m : ops) {
      double dev = 0;
      for (int r = 0; r < 3; ++r) dev += std::abs(m[3 * r] * kq[0] + m[3 * r + 1] * kq[1] + m[3 * r + 2] * kq[2] - kq[r]);
      if (dev <= 1e-9) keep.push_back(m);
    }
    ops.swap(keep);
  }
  // the identity first, then the order of the codes
  const std::array<int, 9> id{1, 0, 0, 0, 1, 0, 0, 0, 1};
  auto itid = std::find(ops.begin(), ops.end(), id);
  if (itid == ops.end()) throw std::runtime_error("symmetry search lost the identity");
  std::rotate(ops.begin(), itid, itid + 1);
  return ops;
}

bool soc_active(const Problem& p) {
  const Material& m = p.mat;
  if (m.use_uniform_us && m.uniform_us != 0.0) return true;
  for (auto& kv : m.Us)
    if (kv.second != 0.0 && !m.use_uniform_us) return true;
  for (auto& kv : m.Ua)
    if (kv.second != 0.0) return true;
  return false;
}

// ----------------------------------------------------------- polarisation vec
// src/pmx_basis.cpp:798-874
void uvec_LT(const Vec3& v0, double out[3][3][2]) {
  Vec3 l = v0;
  if (norm(l) == 0)
    l = {0, 0, 1};
  else
    l = l / norm(l);
  Vec3 t;
  if (v0.y != 0)
    t = {-v0.y, v0.x, 0};
  else if (v0.z != 0)
    t = {v0.z, 0, -v0.x};
  else
    t = {0, 1, 0};
  t = t / norm(t);
  t = t - dot(l, t) * l;
  t = t / norm(t);
  Vec3 pv = cross(l, t);
  pv = pv / norm(pv);
  const double r2 = std::sqrt(2.0);
  for (int x = 0; x < 3; ++x) {
    out[0][x][0] = l[x];
    out[0][x][1] = 0;
    out[1][x][0] = t[x] / r2;
    out[1][x][1] = pv[x] / r2;
    out[2][x][0] = t[x] / r2;
    out[2][x][1] = -pv[x] / r2;
  }
}

// ------------------------------------------------------------------- builder
void build_problem(int argc, const char* const* argv, Problem& p) {
  ArgParser inp(argc, argv);
  p.lat.f = std::sqrt(8.0 / 3.0);
  input_process(inp, p);
  init_crystal(inp, p);
  init_mater(inp, p);
  if (inp.has("-switch")) {
    p.switch_name = inp.value("-switch");
    if (p.switch_name == "band") p.sw = Switch::Band;
    else if (p.switch_name == "epsij") p.sw = Switch::Epsij;
    else if (p.switch_name == "epsLL") p.sw = Switch::EpsLL;
    else if (p.switch_name == "epsxyz") p.sw = Switch::EpsXyz;
  }
  generate_gvectors(p);
  generate_loci(p);
  if (p.kpoint == 0)
    import_kpoints(p);
  else if (p.kpoint == 1)
    generate_kpoints_bz(p);
  else if (p.kpoint == 3)
    generate_kpoints_cohen_chadi(p);
  // kpoint == 2 (Monkhorst-Pack) is an empty stub in the reference
  // (src/pmx_basis.cpp:193-195) and leaves the list empty here too.
}

// -------------------------------------------------------------------- writers
static std::string out_path(const Problem& p, const char* ext) {
  return p.wdir + "/" + p.outputfile + ext;
}

void write_eband(const Problem& p, const std::vector<double>& eband) {
  std::ofstream f(out_path(p, ".dat"), std::ios::binary);
  if (!f) fail("cannot write " + out_path(p, ".dat"));
  f.write(reinterpret_cast<const char*>(eband.data()), eband.size() * sizeof(double));
}

void write_chi(const Problem& p, const std::vector<double>& re, const std::vector<double>& im) {
  std::ofstream f(out_path(p, ".dat"), std::ios::binary);
  if (!f) fail("cannot write " + out_path(p, ".dat"));
  f.write(reinterpret_cast<const char*>(re.data()), re.size() * sizeof(double));
  f.write(reinterpret_cast<const char*>(im.data()), im.size() * sizeof(double));
}

void write_gpt(const Problem& p) {
  std::ofstream f(out_path(p, ".gpt"), std::ios::binary);
  if (!f) fail("cannot write " + out_path(p, ".gpt"));
  for (int g = 0; g < p.neps; ++g)
    for (int i = 0; i < 3; ++i) {
      const double v = p.G[g][i];
      f.write(reinterpret_cast<const char*>(&v), sizeof v);
    }
}

// ----------------------------------------------------------------- text output
void print_doc() {
  std::cout << "============================================================\n"
            << "  PicoMax version 0.1 (B200 build)\n"
            << "Usage:\n"
            << "  picomax [-option] [value]\n"
            << "============================================================\n"
            << "-h, -help : print help\n"
            << "-v, -version : print PicoMax version\n"
            << "-debug : debug level {0}\n"
            << "-outputfile : output filename\n"
            << "-wdir : working directory {pwd}\n"
            << "-logfile : print output to a logfile {0}\n\n"
            << "-switch : calculation switch\n"
            << "    band, epsij, epsLL, epsxyz\n\n"
            << "-crystal : crystal structure\n"
            << "    zb, wz, rs, te, hex\n"
            << "-dim : crystal dimension {3}\n"
            << "-a : lattice constant [angstrom]\n"
            << "-f : lattice parameter\n"
            << "-u : atomic basis parameter\n"
            << "-vg : empirical pseudopotential form factors\n"
            << "-us_so : Symmetric Spin-Orbit form factors (G^2:value,G^2:value,...)\n"
            << "-use_uniform_us_so : Use a single value for symmetric SO coupling for all G^2 (flag)\n"
            << "-uniform_us_so_val : The uniform symmetric SO coupling value in Rydbergs\n"
            << "-ua_so : Antisymmetric Spin-Orbit form factors (G^2:value,G^2:value,...)\n"
            << "-ua_so_val_g0 : Antisymmetric Spin-Orbit form factor for G^2=0 (single value)\n"
            << "-encut : energy cutoff [eV]\n"
            << "-gcut : g-vector cutoff [2*pi/a]\n"
            << "-gsym : spherical (1) or box (0) g-vector grid {1}\n"
            << "-kpoint : switch for kpoint grids\n"
            << "    0->import kpointfile\n"
            << "    1->full BZ\n"
            << "    3->Cohen-Chadi special points\n"
            << "-kpointfile : k-point list file\n"
            << "-kpointorder : kpoint density NxNxN\n"
            << "-nband : number of electronic bands\n"
            << "-neps : the size of dielectric matrix NxN\n"
            << "-nvalence : the number of valence electron bands\n\n"
            << "-qvec : q-vectors\n"
            << "-qpath : path of q-vectors\n"
            << "-qnum : number of q-vectors in each path\n"
            << "-refpoint : the reference q-vector for electronic band energy {0,0,0}\n"
            << "-gammazero : the Gamma-point {0,0,0}\n\n"
            << "-nfreq : number of frequency points {1}\n"
            << "-dfreq : frequency interval [eV]\n"
            << "-delta : delta function model {0}: 0 gaussian, 1 lorentzian, 2 triangle, 3 rect\n"
            << "-epsilon : delta function smearing [eV] {0.1}\n"
            << "-kk : switch for Kramers-Kronig transform {0}\n\n"
            << "B200 options:\n"
            << "-precision : fp64 (default) or mixed (split-BF16 chi contraction)\n"
            << "============================================================\n"
            << std::endl;
}

void print_version() {
  std::cout << "PicoMax version v0.1\n";
  std::cout << "  Date: 2024.06.06 (B200 build)\n";
}

// Eigen prints a row vector with stream precision 6, every entry right-aligned
// to the widest entry and one space between entries; this reproduces the
// `-debug 3` dump lines (src/pmx_io.cpp:572-603).
static std::string row(const Vec3& v) {
  std::string e[3];
  size_t w = 0;
  for (int i = 0; i < 3; ++i) {
    std::ostringstream s;
    s << v[i];
    e[i] = s.str();
    w = std::max(w, e[i].size());
  }
  std::string out;
  for (int i = 0; i < 3; ++i) {
    if (i) out += ' ';
    out += std::string(w - e[i].size(), ' ') + e[i];
  }
  return out;
}

void print_input(const Problem& p) {
  std::cout << "working directory: " << p.wdir << "\n"
            << "outputfile: " << p.outputfile << "\n"
            << "logfile: " << p.logfile << "\n"
            << "number of electronic bands: " << p.nband << "\n"
            << "number of valence electrons: " << p.nvalence << "\n"
            << "size of dielectric matrix: " << p.neps << "\n"
            << "Material properties" << "\n"
            << "lattice constant [angstrom]: " << p.lat.a << "\n"
            << "Empirical pseudopotential form factors, Vg:" << "\n"
            << "g2: \t";
  if (p.mat.NV > 0) {
    for (int i = 0; i < p.mat.NV; ++i) std::cout << p.mat.g2[i] << "\t";
    std::cout << "\n";
    for (int i = 0; i < p.natom; ++i) {
      std::cout << "atom " << (i + 1) << ": ";
      for (int j = 0; j < p.mat.NV; ++j) std::cout << p.mat.vg[i][j] << "\t";
      std::cout << "\n";
    }
  } else {
    std::cout << "(Not provided or not applicable)\n";
  }
  std::cout << "Symmetric Spin-Orbit form factors (Us_SO_Ry):" << "\n";
  if (p.mat.use_uniform_us)
    std::cout << "  Using uniform Us_SO value: " << p.mat.uniform_us << " Ry for all G^2\n";
  else if (!p.mat.Us.empty())
    for (auto& kv : p.mat.Us) std::cout << "  G^2 = " << kv.first << ": " << kv.second << " Ry\n";
  else
    std::cout << "  (Not provided or default values used)\n";
  std::cout << "Antisymmetric Spin-Orbit form factor for G^2=0 (Ua_SO_Ry[0]):" << "\n";
  auto it = p.mat.Ua.find(0);
  if (it != p.mat.Ua.end())
    std::cout << "  G^2 = 0: " << it->second << " Ry\n";
  else
    std::cout << "  (Not provided, effectively 0 for G^2=0 and other G^2 values)\n";
  std::cout << "Antisymmetric Spin-Orbit form factors (Ua_SO_Ry):" << "\n";
  if (!p.mat.Ua.empty())
    for (auto& kv : p.mat.Ua) std::cout << "  G^2 = " << kv.first << ": " << kv.second << " Ry\n";
  else
    std::cout << "  (Not provided or default values used)\n";
  std::cout << "atomic basis vectors:\n";
  for (int i = 0; i < p.natom; ++i) std::cout << " " << row(p.lat.atomic[i]) << "\n";
  std::cout << std::endl;
  std::cout << "planewave energy cutoff [eV]: " << p.lat.encut << std::endl;
  std::cout << "planewave gpoint cutoff [2*pi/a]: " << p.lat.gcut << std::endl;
  std::cout << "number of plane waves: " << p.npw() << std::endl;
  std::cout << "Number of gpoint grids: " << p.npw() << std::endl;
  if (p.debug > 2) {
    for (const Vec3& g : p.G) std::cout << row(g) << "\n";
    std::cout << std::endl;
  }
  if (p.kpoint == 0)
    std::cout << "KPOINT imported from kpointfile: " << p.kpointfile << std::endl;
  else if (p.kpoint == 1)
    std::cout << "KPOINT generated for full BZ with order: " << p.lat.kpointorder << std::endl;
  else if (p.kpoint == 2)
    std::cout << "KPOINT generated for Monkhorst-Pack grids with order: " << p.lat.kpointorder << std::endl;
  else if (p.kpoint == 3)
    std::cout << "KPOINT generated for Cohen-Chadi grids with order: " << p.lat.kpointorder << std::endl;
  std::cout << "Number of K-vector grids: " << p.nk() << std::endl;
  if (p.debug > 2) {
    for (const Vec3& k : p.K) std::cout << row(k) << "\n";
    std::cout << std::endl;
  }
  std::cout << "Number of q-grids: " << p.nq() << std::endl;
  if (p.debug > 2) {
    for (const Vec3& q : p.lat.Q) std::cout << row(q) << "\n";
    std::cout << std::endl;
  }
  for (int i = 0; i < 8; ++i) std::cout << "" << std::endl;
}

}  // namespace pmx
