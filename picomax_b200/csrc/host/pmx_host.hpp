// Host-side problem description for the picomax drop-in: argv grammar, crystal
// presets, form factors, G/k/q tables and the binary writers.
//
// Everything here is plain C++ on the CPU. The GPU stages (pmx_device.hpp) only
// consume the flat tables built here. The integer index tables (G order, loci)
// are bit-exact against the reference (src/pmx_basis.cpp:29-179) because they
// repeat its floating-point sequence and its std::sort call on the same input.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace pmx {

// Physical constants, same values as the reference (src/pmx.hpp:63-71).
constexpr double kPi = 3.14159265358979323846;
constexpr double kHbar = 1.054571817e-27;      // erg s (CGS)
constexpr double kE = 4.803204712570263e-10;   // esu
constexpr double kEm = 9.1093837015e-28;       // g
constexpr double kEV = 1.602176634e-12;        // erg
constexpr double kRy2eV = 13.605699169854621;  // Ry / eV
constexpr double kAngstrom = 1e-8;             // cm
constexpr double kKCON = 3.809982111485962;    // hbar^2/(2 m_e eV A^2)

struct Vec3 {
  double x = 0, y = 0, z = 0;
  double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline Vec3 operator+(const Vec3& a, const Vec3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(const Vec3& a, const Vec3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator*(double s, const Vec3& a) { return {s * a.x, s * a.y, s * a.z}; }
inline Vec3 operator/(const Vec3& a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(const Vec3& a, const Vec3& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double sqnorm(const Vec3& a) { return (a.x * a.x + a.y * a.y) + a.z * a.z; }
double norm(const Vec3& a);
inline Vec3 cross(const Vec3& a, const Vec3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// The reference's inputParser (src/pmx.hpp:190-245): flag = exact token,
// value = next token, first occurrence wins, vectors are comma separated.
class ArgParser {
 public:
  ArgParser(int argc, const char* const* argv);
  bool has(const std::string& opt) const;
  const std::string& value(const std::string& opt) const;
  std::vector<std::string> vec(const std::string& opt) const;
  // Same as inputParser::fill_int/fill_double: std::stoi/std::stod, which throw
  // std::invalid_argument on garbage (the reference terminates there).
  void fill_int(const std::string& opt, int& v) const;
  void fill_double(const std::string& opt, double& v) const;

 private:
  std::vector<std::string> tok_;
};

struct Crystal {
  int dim = 3;
  std::string name;
  std::vector<Vec3> lattice, reciprocal, atomic;
  double a = 0;                  // Angstrom
  double f = 1.6329931618554521;  // sqrt(8/3), set at runtime to sqrt(8.0/3.0)
  double u = 3.0 / 8.0;
  double encut = 200;
  double gcut = 0;
  int gsym = 1;
  int kpointorder = 3;
  double bz_volume = 4;
  std::vector<Vec3> Q;
  std::vector<int> qnum;
  std::vector<std::string> qpath;
  Vec3 gammazero;
};

struct Material {
  int NV = 0;
  double g2max = 0;
  std::vector<double> g2;                // [NV]
  std::vector<std::vector<double>> vg;   // [NATOM][NV] in Ry
  std::map<double, double> Us, Ua;       // SOC maps, key |dG|^2, value Ry
  bool use_uniform_us = false;
  double uniform_us = 0;
};

enum class Switch { None, Band, Epsij, EpsLL, EpsXyz };

// One parsed picomax invocation (src/pmx_io.cpp:108-503).
struct Problem {
  // options
  int debug = 0;
  std::string outputfile = "picomax_output";
  std::string wdir;
  std::string kpointfile;
  int logfile = 0;
  int kpoint = -1;
  int nband = 8;
  int neps = 1;
  int nvalence = 4;
  int nfreq = 1;
  double dfreq = 0;
  bool have_freq = false;
  std::vector<double> freq;
  int kk = 0;
  double epsilon = 0.1;
  int delta = 0;
  Vec3 refpoint;
  Switch sw = Switch::None;
  std::string switch_name;

  Crystal lat;
  Material mat;
  int natom = 0;

  // tables
  std::vector<Vec3> G;                  // [NPW]
  std::vector<std::array<int, 3>> hkl;  // integer coordinates of each G
  int imax = 0;
  std::vector<int> loci;                // [NEPS][NPW]
  std::vector<Vec3> K;                  // [NKPT]
  std::vector<double> KW;               // [NKPT]

  int npw() const { return (int)G.size(); }
  int nk() const { return (int)K.size(); }
  int nq() const { return (int)lat.Q.size(); }
};

// Parse argv exactly as inputProcess/init_crystal/init_mater do, then build the
// G list, loci and the k-point list. Throws std::runtime_error with a message
// where the reference would abort().
void build_problem(int argc, const char* const* argv, Problem& p);

// Individual steps (exposed for tests through the C-ABI).
void generate_gvectors(Problem& p);      // src/pmx_basis.cpp:29-132
void generate_loci(Problem& p);          // src/pmx_basis.cpp:142-179
void import_kpoints(Problem& p);         // src/pmx_basis.cpp:200-245
void generate_kpoints_bz(Problem& p);    // src/pmx_basis.cpp:347-355
void generate_kpoints_cohen_chadi(Problem& p);  // src/pmx_basis.cpp:256-335

// Form factors (src/pmx_epm.cpp:22-50 and :171-203).
double soc_form_factor(const std::map<double, double>& m, double q2);
// Local pseudopotential V(dG) in eV (0 if |dG|^2 >= g2max or no shell match).
void local_potential(const Problem& p, const Vec3& dG, double& re, double& im);
// Spin-orbit scalar VSO(q) = lambda_S cos_sum + i lambda_A sin_sum in eV for
// q = G_j - G_i (src/pmx_epm.cpp:88-118, src/pmx_chi.cpp:203-232).
void soc_scalar(const Problem& p, const Vec3& q, double& re, double& im);
bool soc_active(const Problem& p);

// Point-group operations of the problem's Hamiltonian, as integer matrices M
// in the reciprocal basis (hkl' = M hkl; reduced k coordinates transform the
// same way), row-major. A lattice operation R (|M_ij| <= 1, R orthogonal) is
// kept when some translation t (a difference of atomic positions after R)
// makes the local and spin-orbit form factors over every G difference of the
// basis satisfy V(R dG) = V(dG) exp(-2 pi i R dG . t), and R maps the G list
// onto itself: then H(k) and H(Rk) have the same spectrum. time_reversal adds
// -R for every R (E(-k) = E(k)); little_q keeps only the operations that
// leave q unchanged. The identity comes first.
std::vector<std::array<int, 9>> symmetry_ops(const Problem& p, bool time_reversal, const Vec3* little_q);

// Polarisation vectors [L, (T+iP)/sqrt2, (T-iP)/sqrt2] (src/pmx_basis.cpp:798-874),
// returned as 3 complex 3-vectors: out[i][x] = (re, im).
void uvec_LT(const Vec3& v, double out[3][3][2]);

// Writers (src/pmx_io.cpp:704-826).
void write_eband(const Problem& p, const std::vector<double>& eband);
void write_chi(const Problem& p, const std::vector<double>& re, const std::vector<double>& im);
void write_gpt(const Problem& p);

// Text output mirroring the reference (src/pmx_io.cpp:23-97, :510-614).
void print_doc();
void print_version();
void print_input(const Problem& p);

}  // namespace pmx
