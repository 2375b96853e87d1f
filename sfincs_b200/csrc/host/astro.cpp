// Astronomic water-level boundaries: the .bca reader and the nodal factors.
//
// A .bca file holds one [forcing] block per boundary point, each a list of
// tidal constituents with an amplitude (m) and a phase (degrees)
// (sfincs_boundaries.f90:289-450).  At load the amplitudes are multiplied by
// the nodal factor f of each constituent and the phases reduced by its
// astronomical argument V0+u, both at the reference date tref; each step then
// adds sum A cos(w t - phi) to the level of every boundary point (:736-744).
//
// The nodal factors follow the tidal analysis package that the reference
// vendors (Delft3D astro.f90, `update_nodal_factors` :5-96, `asc` :98-189,
// `hulpgr` :482-643, `datumi` :646-748, `bewvuf` :750-910): the astronomical
// arguments of Schureman's method (mean longitudes of the moon, the sun, the
// lunar perigee and node and the solar perigee, and the node-dependent
// auxiliary angles) from the hours since 1900, and per constituent its
// Doodson-type argument and nodal terms.  The constituent table below holds
// the commonly used constituents with the definitions that package uses;
// a constituent outside it is refused.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "model.h"

namespace sfg {
namespace {

// One tidal constituent: multipliers of the arguments T (mean solar hour
// angle + 180 deg), s, p, h, p1, xi and nu, a phase in quarter turns, up to two
// extra u terms (+-index into the auxiliary angles) and up to three nodal
// factor terms (exponent, index into the auxiliary factors).
struct Constituent {
  const char* name;
  signed char arg[7];
  signed char quarter;
  signed char u[2];
  signed char fexp[3], fidx[3];
};

// Schureman's constituent definitions in the form of the vendored package
// (astro.f90 `kompbs` :192-479, one row per constituent).
const Constituent kConstituents[] = {
    {"SA", {0, 0, 0, 1, 0, 0, 0}, 0, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"SSA", {0, 0, 0, 2, 0, 0, 0}, 0, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"MSM", {0, 1, 1, -2, 0, 0, 0}, 0, {0, 0}, {1, 0, 0}, {1, 0, 0}},
    {"MM", {0, 1, -1, 0, 0, 0, 0}, 0, {0, 0}, {1, 0, 0}, {1, 0, 0}},
    {"MSF", {0, 2, 0, -2, 0, 0, 0}, 0, {0, 0}, {1, 0, 0}, {1, 0, 0}},
    {"MF", {0, 2, 0, 0, 0, -2, 0}, 0, {0, 0}, {1, 0, 0}, {2, 0, 0}},
    {"MFM", {0, 3, -1, 0, 0, -2, 0}, 0, {0, 0}, {1, 0, 0}, {2, 0, 0}},
    {"MSQM", {0, 4, 0, -2, 0, -2, 0}, 0, {0, 0}, {1, 0, 0}, {2, 0, 0}},
    {"MQM", {0, 4, -2, 0, 0, -2, 0}, 0, {0, 0}, {1, 0, 0}, {2, 0, 0}},
    {"2Q1", {1, -4, 2, 1, 0, 2, -1}, 1, {0, 0}, {1, 0, 0}, {3, 0, 0}},
    {"SIGMA1", {1, -4, 0, 3, 0, 2, -1}, 1, {0, 0}, {1, 0, 0}, {3, 0, 0}},
    {"Q1", {1, -3, 1, 1, 0, 2, -1}, 1, {0, 0}, {1, 0, 0}, {3, 0, 0}},
    {"RO1", {1, -3, -1, 3, 0, 2, -1}, 1, {0, 0}, {1, 0, 0}, {3, 0, 0}},
    {"O1", {1, -2, 0, 1, 0, 2, -1}, 1, {0, 0}, {1, 0, 0}, {3, 0, 0}},
    {"M1", {1, -1, 1, 1, 0, 0, -1}, -1, {-12, 0}, {1, 0, 0}, {21, 0, 0}},
    {"NO1", {1, -1, 1, 1, 0, 0, -1}, -1, {0, 0}, {1, 1, 0}, {3, 6, 0}},
    {"PI1", {1, 0, 0, -2, 1, 0, 0}, 1, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"P1", {1, 0, 0, -1, 0, 0, 0}, 1, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"S1", {1, 0, 0, 0, 0, 0, 0}, 0, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"K1", {1, 0, 0, 1, 0, 0, 0}, -1, {-10, 0}, {1, 0, 0}, {19, 0, 0}},
    {"PSI1", {1, 0, 0, 2, -1, 0, 0}, -1, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"FI1", {1, 0, 0, 3, 0, 0, 0}, -1, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"THETA1", {1, 1, 1, -1, 0, 0, -1}, -1, {0, 0}, {1, 0, 0}, {4, 0, 0}},
    {"J1", {1, 1, -1, 1, 0, 0, -1}, -1, {0, 0}, {1, 0, 0}, {4, 0, 0}},
    {"OO1", {1, 2, 0, 1, 0, -2, -1}, -1, {0, 0}, {1, 0, 0}, {5, 0, 0}},
    {"EPSILON2", {2, -5, 1, 4, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"2N2", {2, -4, 2, 2, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"MU2", {2, -4, 0, 4, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"N2", {2, -3, 1, 2, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"NU2", {2, -3, -1, 4, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"M2", {2, -2, 0, 2, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"MKS2", {2, -2, 0, 4, 0, 2, -2}, 0, {-11, 0}, {1, 1, 0}, {6, 20, 0}},
    {"LABDA2", {2, -1, 1, 0, 0, 2, -2}, 2, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"L2", {2, -1, -1, 2, 0, 2, -2}, 2, {-13, 0}, {1, 0, 0}, {22, 0, 0}},
    {"T2", {2, 0, 0, -1, 1, 0, 0}, 0, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"S2", {2, 0, 0, 0, 0, 0, 0}, 0, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"R2", {2, 0, 0, 1, -1, 0, 0}, 2, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"K2", {2, 0, 0, 2, 0, 0, 0}, 0, {-11, 0}, {1, 0, 0}, {20, 0, 0}},
    {"MSN2", {2, 1, -1, 0, 0, 0, 0}, 0, {0, 0}, {2, 0, 0}, {6, 0, 0}},
    {"ETA2", {2, 1, -1, 2, 0, 0, -2}, 0, {0, 0}, {1, 0, 0}, {7, 0, 0}},
    {"2SM2", {2, 2, 0, -2, 0, -2, 2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"MO3", {3, -4, 0, 3, 0, 4, -3}, 1, {0, 0}, {1, 1, 0}, {3, 6, 0}},
    {"2MK3", {3, -4, 0, 3, 0, 4, -4}, 1, {10, 0}, {2, 1, 0}, {6, 19, 0}},
    {"M3", {3, -3, 0, 3, 0, 3, -3}, 0, {0, 0}, {1, 0, 0}, {17, 0, 0}},
    {"MK3", {3, -2, 0, 3, 0, 2, -2}, -1, {-10, 0}, {1, 1, 0}, {6, 19, 0}},
    {"SK3", {3, 0, 0, 1, 0, 0, 0}, -1, {-10, 0}, {1, 0, 0}, {19, 0, 0}},
    {"3MS4", {4, -6, 0, 6, 0, 6, -6}, 0, {0, 0}, {3, 0, 0}, {6, 0, 0}},
    {"MN4", {4, -5, 1, 4, 0, 4, -4}, 0, {0, 0}, {2, 0, 0}, {6, 0, 0}},
    {"M4", {4, -4, 0, 4, 0, 4, -4}, 0, {0, 0}, {2, 0, 0}, {6, 0, 0}},
    {"SN4", {4, -3, 1, 2, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"MS4", {4, -2, 0, 2, 0, 2, -2}, 0, {0, 0}, {1, 0, 0}, {6, 0, 0}},
    {"MK4", {4, -2, 0, 4, 0, 2, -2}, 0, {-11, 0}, {1, 1, 0}, {6, 20, 0}},
    {"S4", {4, 0, 0, 0, 0, 0, 0}, 0, {0, 0}, {0, 0, 0}, {0, 0, 0}},
    {"SK4", {4, 0, 0, 2, 0, 0, 0}, 0, {-11, 0}, {1, 0, 0}, {20, 0, 0}},
    {"2MN6", {6, -7, 1, 6, 0, 6, -6}, 0, {0, 0}, {3, 0, 0}, {6, 0, 0}},
    {"M6", {6, -6, 0, 6, 0, 6, -6}, 0, {0, 0}, {3, 0, 0}, {6, 0, 0}},
    {"2MS6", {6, -4, 0, 4, 0, 4, -4}, 0, {0, 0}, {2, 0, 0}, {6, 0, 0}},
    {"MSK6", {6, -2, 0, 4, 0, 2, -2}, 0, {-11, 0}, {1, 1, 0}, {6, 20, 0}},
    {"M8", {8, -8, 0, 8, 0, 8, -8}, 0, {0, 0}, {4, 0, 0}, {6, 0, 0}},
};

// Fortran MOD(a, p) for reals (the remainder with the sign of a, exact) and
// the "bring into [0, 2 pi)" step of the package: mod(v, 2pi) - 2pi (sign(0.5, v) - 0.5).
double wrap_2pi(double v) {
  const double pix2 = 8.0 * std::atan(1.0);
  const double half = std::signbit(v) ? -0.5 : 0.5;
  return std::fmod(v, pix2) - pix2 * (half - 0.5);
}

// real**integer as the Fortran runtime evaluates it: binary powering.
double powi(double x, int n) {
  double r = 1.0;
  for (unsigned u = (unsigned)n;;) {
    if (u & 1u) r *= x;
    u >>= 1;
    if (u) x *= x;
    else break;
  }
  return r;
}

// Date and time of tref (time_to_vector(0, tref), sfincs_date.f90:329-364): the
// seconds of the day pass through the reference's real*4 fraction of a day.
void tref_vector(const std::string& tref, int v[6]) {
  if (tref.size() < 15) throw std::runtime_error("tref must read yyyymmdd HHMMSS for a bca file");
  const int yyyy = std::atoi(tref.substr(0, 4).c_str()), mm = std::atoi(tref.substr(4, 2).c_str()),
            dd = std::atoi(tref.substr(6, 2).c_str()), hh = std::atoi(tref.substr(9, 2).c_str()),
            mn = std::atoi(tref.substr(11, 2).c_str()), ss = std::atoi(tref.substr(13, 2).c_str());
  const float frac = (float)hh / 24.0f + (float)mn / 1440.0f + (float)ss / 86400.0f;
  const float sec_add = (float)((double)(frac * 86400.0f) + 0.0);
  const int ndays = (int)(sec_add / 86400.0f);
  if (ndays != 0) throw std::runtime_error("tref time of day out of range");
  const float secs = sec_add - (float)ndays * 86400.0f;
  const int h = (int)(secs / 3600.0f);
  const int m = (int)((secs - (float)(h * 3600)) / 60.0f);
  const int s = (int)(secs - (float)(h * 3600) - (float)(m * 60));
  v[0] = yyyy, v[1] = mm, v[2] = dd, v[3] = h, v[4] = m, v[5] = s;
}

// Hours since January 1, 00:00 of the date's own year (astro.f90 `datumi` :646-748).
double hours_in_year(const int d[6]) {
  static const double cum[12] = {0, 31, 59, 90, 120, 151, 181, 212, 243, 273, 304, 334};
  if (d[1] < 1 || d[1] > 12) throw std::runtime_error("tref month out of range");
  double days = cum[d[1] - 1];
  const bool leap = d[0] % 4 == 0 && (d[0] % 100 != 0 || d[0] % 400 == 0);
  if (leap && d[1] >= 3) days += 1.0;
  return days * 24.0 + (double)(float)(d[2] - 1) * 24.0 + (double)(float)d[3] + (double)(float)d[4] / 60.0 +
         (double)(float)d[5] / 3600.0;
}

// Auxiliary angles v[1..15] (rad) and factors f[1..22] (astro.f90 `hulpgr` :482-643).
void auxiliary(int year, double hours, double v[16], double f[26]) {
  const double pix2 = 8.0 * std::atan(1.0), rad = pix2 / 360.0;
  const double ry = (double)(float)(year - 1900);
  const int leapdays = (int)((ry - 0.99) / 4.0) - (int)((ry - 0.99) / 100.0) + (int)((ry + 300.0 - 0.99) / 400.0);
  const double d = (double)(float)leapdays + hours / 24.0;
  v[1] = (180.000 + 360.0000000 * d) * rad;
  v[2] = (277.026 + 129.3848200 * ry + 13.176396800000 * d) * rad;
  v[3] = (334.384 + 40.6624700 * ry + 0.111404000000 * d) * rad;
  v[4] = (280.190 - 0.2387136 * ry + 0.985647360000 * d) * rad;
  v[5] = (281.221 + 0.0171800 * ry + 0.000047064943 * d) * rad;
  v[8] = (259.156 + 340.6718100 * ry - 0.052953945000 * d) * rad;
  double z = 0.009415;
  const double a1 = std::atan(z * std::sin(v[8]) / (1.0 + z * (1.0 - std::cos(v[8]))));
  z = -0.17794;
  const double a2 = std::atan(z * std::sin(v[8]) / (1.0 + z * (1.0 - std::cos(v[8]))));
  v[6] = -a1 - a2;
  v[7] = a1 - a2;
  const double rk0 = 0.9137 - 0.03569 * std::cos(v[8]);
  const double ri = std::atan(std::sqrt(1.0 - rk0 * rk0) / rk0);
  v[9] = ri;
  const double per = wrap_2pi(v[3]);
  const double xi = v[6], nu = v[7];
  const double s2ri = std::sin(2.0 * ri), sri = std::sin(ri), si = std::sin(0.5 * ri), cri = std::cos(ri),
               ci = std::cos(0.5 * ri);
  v[10] = std::atan(s2ri * std::sin(nu) / (s2ri * std::cos(nu) + 0.3347));
  v[11] = std::atan(sri * sri * std::sin(2.0 * nu) / (sri * sri * std::cos(2.0 * nu) + 0.0727));
  v[12] = std::atan(std::sin(2.0 * (per - xi)) / (3.0 * cri / (ci * ci) + std::cos(2.0 * (per - xi))));
  v[13] = std::atan(std::sin(2.0 * (per - xi)) / (ci * ci / (si * si * 6.0) - std::cos(2.0 * (per - xi))));
  v[14] = 3.0 * v[10];
  v[15] = 0.0;
  for (int j = 1; j <= 15; j++) v[j] = wrap_2pi(v[j]);
  const double ci4 = ci * ci * ci * ci, si4 = si * si * si * si, sri3 = sri * sri * sri;
  f[1] = (2.0 / 3.0 - sri * sri) / 0.5021;
  f[2] = sri * sri / 0.1578;
  f[3] = sri * ci * ci / 0.38;
  f[4] = s2ri / 0.7214;
  f[5] = sri * si * si / 0.0164;
  f[6] = ci4 / 0.9154;
  f[7] = sri * sri / 0.1565;
  f[8] = si4 / 0.0017;
  f[9] = (sri - 1.25 * sri3) / 0.3192;
  f[10] = sri3 / 0.063;
  f[11] = sri * sri * ci * ci / 0.1518;
  f[12] = (1.0 - 10.0 * si * si + 15.0 * si4) * ci * ci / 0.5873;
  f[13] = (1.0 - 10.0 * ci * ci + 15.0 * ci4) * si * si / 0.2147;
  f[14] = sri * ci4 / 0.3658;
  f[15] = (ci * ci - 2.0 / 3.0) * sri * ci * ci / 0.1114;
  f[16] = (ci * ci - 1.0 / 3.0) * sri * si * si / 0.0103;
  f[17] = ci4 * ci * ci / 0.8758;
  f[18] = ci4 * si * si / 0.038;
  f[19] = std::sqrt(0.8965 * s2ri * s2ri + 0.6001 * s2ri * std::cos(nu) + 0.1006);
  f[20] = std::sqrt(19.0444 * sri3 * sri + 2.7702 * sri * sri * std::cos(2.0 * nu) + 0.0981);
  f[21] = 6.0 * cri * std::cos(2.0 * (per - xi)) / (ci * ci) + 9.0 * cri * cri / ci4;
  f[21] = 2.6316 * sri * ci * ci * 0.5 * std::sqrt(1.0 + f[21]);
  f[22] = 36.0 * si4 / ci4 - 12.0 * si * si / (ci * ci) * std::cos(2.0 * (per - xi));
  f[22] = 1.0924 * ci4 * std::sqrt(1.0 + f[22]);
}

std::string clean(const std::string& s) {
  std::string o = s;
  const size_t cr = o.find('\r');
  if (cr != std::string::npos) o = o.substr(0, cr);
  const size_t a = o.find_first_not_of(" \t");
  if (a == std::string::npos) return "";
  o = o.substr(a);
  const size_t b = o.find_last_not_of(" \t");
  return o.substr(0, b + 1);
}

bool is_meta(const std::string& l) {
  for (const char* k : {"Quantity", "Unit", "Name", "Function", "quantity", "unit", "name", "function"})
    if (l.find(k) != std::string::npos) return true;
  return false;
}

// A data line: a name and two reals, separated by blanks or commas.
bool data_line(const std::string& l, std::string& name, float& a, float& p) {
  std::string s = l;
  for (char& c : s)
    if (c == ',' || c == '\t') c = ' ';
  std::istringstream is(s);
  std::string ta, tp;
  if (!(is >> name >> ta >> tp)) return false;
  char* e = nullptr;
  a = std::strtof(ta.c_str(), &e);
  if (e == ta.c_str() || *e) return false;
  p = std::strtof(tp.c_str(), &e);
  if (e == tp.c_str() || *e) return false;
  return true;
}

}  // namespace

// sfincs_boundaries.f90:289-450 with astro.f90 :5-96.
void read_bca_file(const std::string& file, const std::string& tref, int nbnd, TideHost& out) {
  std::ifstream in(file);
  if (!in) throw std::runtime_error("cannot open bca file " + file);
  std::vector<std::string> lines;
  for (std::string l; std::getline(in, l);) lines.push_back(clean(l));
  // first pass: sets, components of the first set, whether it starts with A0
  int nsets = 0, ncomp = 0;
  bool has_a0 = false;
  for (const auto& l : lines) {
    std::string nm;
    float a, p;
    if (l == "[forcing]" || l == "[Forcing]") {
      nsets++;
    } else if (!is_meta(l) && data_line(l, nm, a, p)) {
      if (nsets == 0) throw std::runtime_error("bca file: a constituent line before the first [forcing] block");
      if (nsets == 1) {
        ncomp++;
        if (ncomp == 1 && (nm.compare(0, 2, "a0") == 0 || nm.compare(0, 2, "A0") == 0)) has_a0 = true;
      }
    }
  }
  if (nsets != nbnd)
    throw std::runtime_error("bca file has " + std::to_string(nsets) + " [forcing] blocks for " +
                             std::to_string(nbnd) + " boundary points");
  if (!has_a0) ncomp++;
  // second pass: names (the last block to write a position names it), amplitude and phase per point
  std::vector<std::string> names(ncomp);
  std::vector<double> amp((size_t)ncomp * nbnd, 0.0), pha((size_t)ncomp * nbnd, 0.0);
  int set = 0, k = 0;
  for (const auto& l : lines) {
    std::string nm;
    float a, p;
    if (l == "[forcing]" || l == "[Forcing]") {
      set++;
      k = 0;
      if (!has_a0) names[0] = "A0", k = 1;
    } else if (!is_meta(l) && data_line(l, nm, a, p)) {
      if (k >= ncomp) throw std::runtime_error("bca file: block " + std::to_string(set) + " has more constituents than the first");
      if (nm.size() > 8) throw std::runtime_error("bca file: constituent name longer than 8 characters: " + nm);
      names[k] = nm;
      amp[(size_t)(set - 1) * ncomp + k] = (double)a;
      pha[(size_t)(set - 1) * ncomp + k] = (double)p;
      k++;
    }
  }
  // nodal factors at tref (update_nodal_factors, asc, datumi, hulpgr, bewvuf)
  int d[6];
  tref_vector(tref, d);
  double v[16] = {0}, f[26] = {0};
  auxiliary(d[0], hours_in_year(d), v, f);
  const double pi = (double)(4.0f * std::atan(1.0f));  // the package's single-precision pi
  const double pix2 = 8.0 * std::atan(1.0);
  out.ncomp = ncomp;
  out.names = names;
  out.omega.assign(ncomp, 0.0);  // A0 (first): the package leaves its frequency unset; taken as 0
  for (int c = 1; c < ncomp; c++) {
    std::string nm = names[c];
    if (nm == "EPS2") nm = "EPSILON2";
    if (nm == "LA2") nm = "LABDA2";
    if (nm == "MTM") nm = "MFM";
    const Constituent* kc = nullptr;
    for (const auto& q : kConstituents)
      if (nm == q.name) kc = &q;
    if (!kc) throw std::runtime_error("bca file: tidal constituent '" + names[c] + "' is not in this core's table");
    const double speed = (double)kc->arg[0] * 15.0 + (double)kc->arg[1] * 0.54901653 +
                         (double)kc->arg[2] * 0.0046418333 + (double)kc->arg[3] * 0.04106864 +
                         (double)kc->arg[4] * 0.0000019610393;  // deg/h
    const double w = speed * pix2 / 360.0;                       // rad/h
    double v0u = ((double)kc->quarter * pix2) / 4.0;
    for (int j = 0; j < 7; j++) v0u = v0u + v[j + 1] * (double)kc->arg[j];
    for (int j = 0; j < 2 && kc->u[j] != 0; j++) {
      const int ia = std::abs((int)kc->u[j]);
      v0u = v0u + (kc->u[j] > 0 ? 1.0 : -1.0) * v[ia];
    }
    v0u = wrap_2pi(v0u);
    double fr = 1.0;
    for (int j = 0; j < 3 && kc->fexp[j] != 0; j++) fr = j == 0 ? powi(f[kc->fidx[j]], kc->fexp[j])
                                                              : fr * powi(f[kc->fidx[j]], kc->fexp[j]);
    out.omega[c] = w / 3600.0;  // rad/s
    for (int ib = 0; ib < nbnd; ib++) {
      double& A = amp[(size_t)ib * ncomp + c];
      double& P = pha[(size_t)ib * ncomp + c];
      A = A * fr;
      P = (pi / 180.0) * P - v0u;
      // Fortran MODULO(P, 2 pi): the remainder with the sign of 2 pi
      const double twopi = 2.0 * pi;
      double r = std::fmod(P, twopi);
      if (r != 0.0 && r < 0.0) r += twopi;
      P = r;
    }
  }
  out.amp = amp;
  out.phase = pha;
}

}  // namespace sfg
