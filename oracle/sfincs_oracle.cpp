// SFINCS time-stepping oracle: a CPU restatement of the reference's hot path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
// calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg use it, as the checker.
//
// Parity status: UNPINNED against reference outputs.  The reference (Fortran 90
// + netcdf-fortran) cannot be compiled in this image (no Fortran compiler, no
// netCDF-C library) and ships no tests or golden vectors; this restatement is
// pinned by analytic invariants and hand-derived single-step known answers in
// tests/ instead.
//
// The code mirrors the reference routine by routine, with 1-based arrays so the
// index arithmetic reads like the Fortran.  Every function names the reference
// lines it restates (paths relative to the SFINCS source tree).
//
// Precision is a template parameter: T for the reference's real*4 quantities,
// TZ for zs (real*8 in the reference), TV for z_volume (real*8).  Three
// instantiations are exported: "fp64" (everything double), "ref" (the
// reference's own mixed precision) and "f32" (the CUDA core's precision: zs in
// float, z_volume in double).  Build with -ffp-contract=off so float
// expressions round exactly as written.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <type_traits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "ncread.h"

namespace orc {

template <class X>
struct F1 {  // 1-based Fortran-style vector
  std::vector<X> v;
  void alloc(long n, X init = X(0)) { v.assign((size_t)n + 1, init); }
  X& operator()(long i) { return v[(size_t)i]; }
  const X& operator()(long i) const { return v[(size_t)i]; }
  long size() const { return v.empty() ? 0 : (long)v.size() - 1; }
  bool allocated() const { return !v.empty(); }
  void fill(X x) { std::fill(v.begin() + (v.empty() ? 0 : 1), v.end(), x); }
};

// Cube root of the core-precision ("f32") instantiation, restating the CUDA
// core's method with the same IEEE operations in the same order, so both give
// the same bits: an estimate of x^(-1/3) from the float's bit pattern
// (0x54a232a0 - bits / 3), two Newton steps r += r (1 - x r^3) / 3, y = x r^2
// and one Newton correction of y; denormals are scaled by 2^72 first.  The
// "ref" and "fp64" instantiations keep the reference's power x**(1.0/3.0).
static float core_cube_root_pos(float x) {
  float s = 1.0f;
  if (x < 1.17549435e-38f) {
    x = x * 4722366482869645213696.0f;
    s = 5.9604644775390625e-08f;
  }
  uint32_t bits;
  std::memcpy(&bits, &x, 4);
  bits = 0x54a232a0u - bits / 3u;
  float r;
  std::memcpy(&r, &bits, 4);
  for (int k = 0; k < 2; k++) {
    const float r3 = (r * r) * r;
    const float e = std::fma(-x, r3, 1.0f);
    r = std::fma(r * 0.333333343f, e, r);
  }
  float y = (x * r) * r;
  const float res = std::fma(-(y * y), y, x);
  y = std::fma(res * 0.333333343f, r * r, y);
  return y * s;
}
static float core_cube_root(float x) {
  if (x > 0.0f && x < 3.40282347e+38f) return core_cube_root_pos(x);
  if (x < 0.0f && x > -3.40282347e+38f) return -core_cube_root_pos(-x);
  return x + x;
}

// Four-quadrant arctangent in IEEE operations (the core's own: argument
// reduction by atan(a) = pi/6 + atan((sqrt3 a - 1)/(sqrt3 + a)) above
// tan(pi/12), then the Taylor series to degree 15).
static float core_atan2(float y, float x) {
  const float ax = std::fabs(x), ay = std::fabs(y);
  const float mx = std::max(ax, ay), mn = std::min(ax, ay);
  if (mx == 0.0f) return 0.0f;
  const float a = mn / mx;
  float t = a, off = 0.0f;
  if (a > 0.267949194f) {
    t = (1.73205081f * a - 1.0f) / (1.73205081f + a);
    off = 0.523598776f;
  }
  const float t2 = t * t;
  const float c[6] = {1.0f / 13.0f, -1.0f / 11.0f, 1.0f / 9.0f, -1.0f / 7.0f, 1.0f / 5.0f, -1.0f / 3.0f};
  float p = -1.0f / 15.0f;
  for (int k = 0; k < 6; k++) p = std::fma(p, t2, c[k]);
  float r = off + std::fma(t * t2, p, t);
  if (ay > ax) r = 1.57079633f - r;
  if (x < 0.0f) r = 3.14159265f - r;
  return y < 0.0f ? -r : r;
}


// Exponential of the core-precision instantiation (Horton infiltration),
// restating the CUDA core's method with the same IEEE operations: n =
// rint(x log2 e), r = x - n ln2 with ln2 split in two parts (Cody and Waite),
// e^r by its Taylor polynomial to degree 7 in Horner form with fused
// multiply-adds, times 2^n in two factors.
static float core_exp(float x) {
  if (x != x) return x;
  if (x > 88.8f) return INFINITY;
  if (x < -104.0f) return 0.0f;
  const float n = std::nearbyint(x * 1.44269502f);
  float r = std::fma(-n, 0.693145752f, x);
  r = std::fma(-n, 1.42860677e-06f, r);
  float p = 1.98412701e-04f;  // 1/5040
  p = std::fma(p, r, 1.38888892e-03f);  // 1/720
  p = std::fma(p, r, 8.33333377e-03f);  // 1/120
  p = std::fma(p, r, 4.16666679e-02f);  // 1/24
  p = std::fma(p, r, 1.66666672e-01f);  // 1/6
  p = std::fma(p, r, 0.5f);
  p = std::fma(p, r, 1.0f);
  p = std::fma(p, r, 1.0f);
  const int ni = (int)n, n1 = ni / 2, n2 = ni - n1;
  auto pow2 = [](int e) {
    uint32_t b = (uint32_t)(e + 127) << 23;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
  };
  return (p * pow2(n1)) * pow2(n2);
}

// Cosine in FP64 of the core-precision instantiation (astronomic boundary
// constituents), restating the CUDA core's method with the same IEEE
// operations: n = rint(x 2/pi), r = x - n pi/2 with pi/2 split in three
// doubles, each product fused with its subtraction (Cody and Waite), then the
// Taylor series of sin (degree 17) or cos (degree 18) of r in Horner form with
// fused multiply-adds, by the quadrant n mod 4.  The "ref" and "fp64"
// instantiations call the library cosine, as the reference does.
static double core_cos(double x) {
  const double n = std::nearbyint(x * 0.6366197723675814);
  double r = std::fma(-n, 1.5707963267948966, x);
  r = std::fma(-n, 6.123233995736766e-17, r);
  r = std::fma(-n, -1.4973849048591698e-33, r);
  const double r2 = r * r;
  const int q = (int)((long long)n & 3);
  if (q & 1) {
    const double c[8] = {2.8114572543455206e-15, -7.647163731819816e-13, 1.6059043836821613e-10,
                         -2.505210838544172e-08,  2.7557319223985893e-06, -0.0001984126984126984,
                         0.008333333333333333,    -0.16666666666666666};
    double p = c[0];
    for (int k = 1; k < 8; k++) p = std::fma(p, r2, c[k]);
    const double sn = std::fma(r * r2, p, r);
    return q == 1 ? -sn : sn;
  }
  const double c[9] = {-1.5619206968586225e-16, 4.779477332387385e-14, -1.1470745597729725e-11,
                       2.08767569878681e-09,    -2.755731922398589e-07, 2.48015873015873e-05,
                       -0.001388888888888889,   0.041666666666666664,   -0.5};
  double p = c[0];
  for (int k = 1; k < 9; k++) p = std::fma(p, r2, c[k]);
  const double cs = std::fma(r2, p, 1.0);
  return q == 0 ? cs : -cs;
}

// ------------------------------------------------------- astronomic constituents
// The nodal factors of the tidal package the reference vendors (Delft3D
// astro.f90): `update_nodal_factors` :5-96, `asc` :98-189, `hulpgr`
// :482-643, `datumi` :646-748, `bewvuf` :750-910.  Per constituent: the
// multipliers of v(1..7) (T, s, p, h, p1, xi, nu), the phase in quarter turns
// (field 8), two extra u terms (+-index into v) and three (exponent, index
// into f) nodal factor terms, for the constituents of `kompbs` :192-479 this
// oracle carries.
struct AstroRow {
  const char* name;
  int j[16];
};
static const AstroRow kAstro[] = {
    {"SA", {0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"SSA", {0, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"MSM", {0, 1, 1, -2, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 0}},
    {"MM", {0, 1, -1, 0, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 0}},
    {"MSF", {0, 2, 0, -2, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 0}},
    {"MF", {0, 2, 0, 0, 0, -2, 0, 0, 0, 0, 1, 2, 0, 0, 0, 0}},
    {"MFM", {0, 3, -1, 0, 0, -2, 0, 0, 0, 0, 1, 2, 0, 0, 0, 0}},
    {"MSQM", {0, 4, 0, -2, 0, -2, 0, 0, 0, 0, 1, 2, 0, 0, 0, 0}},
    {"MQM", {0, 4, -2, 0, 0, -2, 0, 0, 0, 0, 1, 2, 0, 0, 0, 0}},
    {"2Q1", {1, -4, 2, 1, 0, 2, -1, 1, 0, 0, 1, 3, 0, 0, 0, 0}},
    {"SIGMA1", {1, -4, 0, 3, 0, 2, -1, 1, 0, 0, 1, 3, 0, 0, 0, 0}},
    {"Q1", {1, -3, 1, 1, 0, 2, -1, 1, 0, 0, 1, 3, 0, 0, 0, 0}},
    {"RO1", {1, -3, -1, 3, 0, 2, -1, 1, 0, 0, 1, 3, 0, 0, 0, 0}},
    {"O1", {1, -2, 0, 1, 0, 2, -1, 1, 0, 0, 1, 3, 0, 0, 0, 0}},
    {"M1", {1, -1, 1, 1, 0, 0, -1, -1, -12, 0, 1, 21, 0, 0, 0, 0}},
    {"NO1", {1, -1, 1, 1, 0, 0, -1, -1, 0, 0, 1, 3, 1, 6, 0, 0}},
    {"PI1", {1, 0, 0, -2, 1, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"P1", {1, 0, 0, -1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"S1", {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"K1", {1, 0, 0, 1, 0, 0, 0, -1, -10, 0, 1, 19, 0, 0, 0, 0}},
    {"PSI1", {1, 0, 0, 2, -1, 0, 0, -1, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"FI1", {1, 0, 0, 3, 0, 0, 0, -1, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"THETA1", {1, 1, 1, -1, 0, 0, -1, -1, 0, 0, 1, 4, 0, 0, 0, 0}},
    {"J1", {1, 1, -1, 1, 0, 0, -1, -1, 0, 0, 1, 4, 0, 0, 0, 0}},
    {"OO1", {1, 2, 0, 1, 0, -2, -1, -1, 0, 0, 1, 5, 0, 0, 0, 0}},
    {"EPSILON2", {2, -5, 1, 4, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"2N2", {2, -4, 2, 2, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"MU2", {2, -4, 0, 4, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"N2", {2, -3, 1, 2, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"NU2", {2, -3, -1, 4, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"M2", {2, -2, 0, 2, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"MKS2", {2, -2, 0, 4, 0, 2, -2, 0, -11, 0, 1, 6, 1, 20, 0, 0}},
    {"LABDA2", {2, -1, 1, 0, 0, 2, -2, 2, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"L2", {2, -1, -1, 2, 0, 2, -2, 2, -13, 0, 1, 22, 0, 0, 0, 0}},
    {"T2", {2, 0, 0, -1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"S2", {2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"R2", {2, 0, 0, 1, -1, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"K2", {2, 0, 0, 2, 0, 0, 0, 0, -11, 0, 1, 20, 0, 0, 0, 0}},
    {"MSN2", {2, 1, -1, 0, 0, 0, 0, 0, 0, 0, 2, 6, 0, 0, 0, 0}},
    {"ETA2", {2, 1, -1, 2, 0, 0, -2, 0, 0, 0, 1, 7, 0, 0, 0, 0}},
    {"2SM2", {2, 2, 0, -2, 0, -2, 2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"MO3", {3, -4, 0, 3, 0, 4, -3, 1, 0, 0, 1, 3, 1, 6, 0, 0}},
    {"2MK3", {3, -4, 0, 3, 0, 4, -4, 1, 10, 0, 2, 6, 1, 19, 0, 0}},
    {"M3", {3, -3, 0, 3, 0, 3, -3, 0, 0, 0, 1, 17, 0, 0, 0, 0}},
    {"MK3", {3, -2, 0, 3, 0, 2, -2, -1, -10, 0, 1, 6, 1, 19, 0, 0}},
    {"SK3", {3, 0, 0, 1, 0, 0, 0, -1, -10, 0, 1, 19, 0, 0, 0, 0}},
    {"3MS4", {4, -6, 0, 6, 0, 6, -6, 0, 0, 0, 3, 6, 0, 0, 0, 0}},
    {"MN4", {4, -5, 1, 4, 0, 4, -4, 0, 0, 0, 2, 6, 0, 0, 0, 0}},
    {"M4", {4, -4, 0, 4, 0, 4, -4, 0, 0, 0, 2, 6, 0, 0, 0, 0}},
    {"SN4", {4, -3, 1, 2, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"MS4", {4, -2, 0, 2, 0, 2, -2, 0, 0, 0, 1, 6, 0, 0, 0, 0}},
    {"MK4", {4, -2, 0, 4, 0, 2, -2, 0, -11, 0, 1, 6, 1, 20, 0, 0}},
    {"S4", {4, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {"SK4", {4, 0, 0, 2, 0, 0, 0, 0, -11, 0, 1, 20, 0, 0, 0, 0}},
    {"2MN6", {6, -7, 1, 6, 0, 6, -6, 0, 0, 0, 3, 6, 0, 0, 0, 0}},
    {"M6", {6, -6, 0, 6, 0, 6, -6, 0, 0, 0, 3, 6, 0, 0, 0, 0}},
    {"2MS6", {6, -4, 0, 4, 0, 4, -4, 0, 0, 0, 2, 6, 0, 0, 0, 0}},
    {"MSK6", {6, -2, 0, 4, 0, 2, -2, 0, -11, 0, 1, 6, 1, 20, 0, 0}},
    {"M8", {8, -8, 0, 8, 0, 8, -8, 0, 0, 0, 4, 6, 0, 0, 0, 0}},
};

// Fortran SIGN(0.5d0, v) (negative zero counts as negative) and MOD for reals.
static double fsign_half(double v) { return std::signbit(v) ? -0.5 : 0.5; }
static double fpowi(double x, int n) {  // real**integer by binary powering (the Fortran runtime)
  double r = 1.0;
  for (unsigned u = (unsigned)n;;) {
    if (u & 1u) r *= x;
    u >>= 1;
    if (u) x *= x;
    else break;
  }
  return r;
}

// hulpgr (astro.f90:482-643): v(1..15), f(1..22) for year jaar and tm1 hours into it.
static void astro_hulpgr(int jaar, double tm1, double* v, double* f) {
  const double pix2 = 8.0 * std::atan(1.0), dhalf = 0.5, rad = pix2 / 360.0;
  const double rjaar = (double)(float)(jaar - 1900);
  const int ischrk = (int)((rjaar - 0.99) / 4.0) - (int)((rjaar - 0.99) / 100.0) + (int)((rjaar + 300.0 - 0.99) / 400.0);
  const double tm3 = (double)(float)ischrk + tm1 / 24.0;
  v[1] = (180.000 + 360.0000000 * tm3) * rad;
  v[2] = (277.026 + 129.3848200 * rjaar + 13.176396800000 * tm3) * rad;
  v[3] = (334.384 + 40.6624700 * rjaar + 0.111404000000 * tm3) * rad;
  v[4] = (280.190 - 0.2387136 * rjaar + 0.985647360000 * tm3) * rad;
  v[5] = (281.221 + 0.0171800 * rjaar + 0.000047064943 * tm3) * rad;
  v[8] = (259.156 + 340.6718100 * rjaar - 0.052953945000 * tm3) * rad;
  double z = 0.009415;
  double p = std::atan(z * std::sin(v[8]) / (1.0 + z * (1.0 - std::cos(v[8]))));
  z = -0.17794;
  const double q = std::atan(z * std::sin(v[8]) / (1.0 + z * (1.0 - std::cos(v[8]))));
  v[6] = -p - q;
  v[7] = p - q;
  double rk = 0.9137 - 0.03569 * std::cos(v[8]);
  const double ri = std::atan(std::sqrt(1.0 - rk * rk) / rk);
  v[9] = ri;
  p = std::fmod(v[3], pix2) - pix2 * (fsign_half(v[3]) - dhalf);
  rk = v[6];
  const double rn1 = v[7];
  const double s2ri = std::sin(2.0 * ri), sri = std::sin(ri), si = std::sin(0.5 * ri), cri = std::cos(ri),
               ci = std::cos(0.5 * ri);
  v[10] = std::atan(s2ri * std::sin(rn1) / (s2ri * std::cos(rn1) + 0.3347));
  v[11] = std::atan(sri * sri * std::sin(2.0 * rn1) / (sri * sri * std::cos(2.0 * rn1) + 0.0727));
  v[12] = std::atan(std::sin(2.0 * (p - rk)) / (3.0 * cri / (ci * ci) + std::cos(2.0 * (p - rk))));
  v[13] = std::atan(std::sin(2.0 * (p - rk)) / (ci * ci / (si * si * 6.0) - std::cos(2.0 * (p - rk))));
  v[14] = 3.0 * v[10];
  v[15] = 0.0;
  for (int j = 1; j <= 15; j++) v[j] = std::fmod(v[j], pix2) - pix2 * (fsign_half(v[j]) - dhalf);
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
  f[19] = std::sqrt(0.8965 * s2ri * s2ri + 0.6001 * s2ri * std::cos(rn1) + 0.1006);
  f[20] = std::sqrt(19.0444 * sri3 * sri + 2.7702 * sri * sri * std::cos(2.0 * rn1) + 0.0981);
  f[21] = 6.0 * cri * std::cos(2.0 * (p - rk)) / (ci * ci) + 9.0 * cri * cri / (ci4);
  f[21] = 2.6316 * sri * ci * ci * 0.5 * std::sqrt(1.0 + f[21]);
  f[22] = 36.0 * si4 / (ci4) - 12.0 * si * si / (ci * ci) * std::cos(2.0 * (p - rk));
  f[22] = 1.0924 * ci4 * std::sqrt(1.0 + f[22]);
}

// bewvuf (astro.f90:750-910) for one constituent: w (rad/h), v0u (rad), fr.
static bool astro_bewvuf(const std::string& name, const double* v, const double* f, double& w, double& v0u,
                         double& fr) {
  const double pix2 = 8.0 * std::atan(1.0), dhalf = 0.5;
  for (const auto& row : kAstro) {
    if (name != row.name) continue;
    const int* jn = row.j;
    w = (double)jn[0] * 15.0 + (double)jn[1] * 0.54901653 + (double)jn[2] * 0.0046418333 +
        (double)jn[3] * 0.04106864 + (double)jn[4] * 0.0000019610393;
    w = (w * pix2) / 360.0;
    v0u = ((double)jn[7] * pix2) / 4.0;
    for (int kw = 1; kw <= 7; kw++) v0u = v0u + v[kw] * (double)jn[kw - 1];
    const int ie1 = jn[8];
    if (ie1 != 0) {
      const int ia1 = std::abs(ie1);
      v0u = v0u + (double)(float)(ie1 / ia1) * v[ia1];
      const int ie2 = jn[9];
      if (ie2 != 0) {
        const int ia2 = std::abs(ie2);
        v0u = v0u + (double)(float)(ie2 / ia2) * v[ia2];
      }
    }
    v0u = std::fmod(v0u, pix2) - pix2 * (fsign_half(v0u) - dhalf);
    fr = 1.0;
    if (jn[10] != 0) {
      fr = fpowi(f[jn[11]], jn[10]);
      if (jn[12] != 0) {
        fr = fr * fpowi(f[jn[13]], jn[12]);
        if (jn[14] != 0) fr = fr * fpowi(f[jn[15]], jn[14]);
      }
    }
    return true;
  }
  return false;
}

template <class X>
struct F2 {  // (n1, n2) column-major, 1-based
  std::vector<X> v;
  long n1 = 0, n2 = 0;
  void alloc(long a, long b, X init = X(0)) { n1 = a; n2 = b; v.assign((size_t)a * b, init); }
  X& operator()(long i, long j) { return v[(size_t)(j - 1) * n1 + (i - 1)]; }
};

// ----------------------------------------------------------------- sfincs.inp
// read_line / read_*_input: sfincs_read.f90:5-249.
struct InpFile {
  std::vector<std::pair<std::string, std::string>> kv;
  explicit InpFile(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::string line0;
    while (std::getline(f, line0)) {
      // notabs: tab stops every 8 columns (sfincs_read.f90:252-300)
      std::string line;
      for (char c : line0) {
        if (c == '\t') {
          size_t ip = line.size() + 1;
          ip = ip + (8 - ((ip - 1) % 8));
          line.resize(ip - 1, ' ');
        } else {
          line.push_back(c);
        }
      }
      size_t jn = line.find('\r');
      if (jn != std::string::npos) line = line.substr(0, jn);
      if (line.empty()) continue;
      if (line[0] == '#' || line[0] == '!' || line[0] == '@') continue;
      size_t j = line.find('=');
      if (j == std::string::npos) continue;
      std::string key = line.substr(0, j);
      while (!key.empty() && key.back() == ' ') key.pop_back();
      std::string val = line.substr(j + 1);
      size_t h = val.find('#');
      if (h != std::string::npos) val = val.substr(0, h);
      size_t a = val.find_first_not_of(' ');
      val = (a == std::string::npos) ? std::string() : val.substr(a);
      while (!val.empty() && val.back() == ' ') val.pop_back();
      kv.emplace_back(key, val);
    }
  }
  const std::string* find(const std::string& key) const {
    for (auto& p : kv)
      if (p.first == key) return &p.second;
    return nullptr;
  }
  float real(const std::string& k, float def) const {
    auto s = find(k);
    return s ? (float)std::strtod(s->c_str(), nullptr) : def;
  }
  int integer(const std::string& k, int def) const {
    auto s = find(k);
    return s ? (int)std::strtol(s->c_str(), nullptr, 10) : def;
  }
  std::string str(const std::string& k, const std::string& def) const {
    auto s = find(k);
    return s ? *s : def;
  }
  bool logical(const std::string& k, bool def) const {
    auto s = find(k);
    if (!s) return def;
    char c = s->empty() ? ' ' : (*s)[0];
    return c == '1' || c == 'y' || c == 'Y' || c == 't' || c == 'T';
  }
};

// julian_date / time_difference: sfincs_date.f90:183-215
static long julian_date(long y, long m, long d) {
  return d - 32075 + 1461 * (y + 4800 + (m - 14) / 12) / 4 + 367 * (m - 2 - ((m - 14) / 12) * 12) / 12 -
         3 * ((y + 4900 + (m - 14) / 12) / 100) / 4;
}
static long time_difference(const std::string& a, const std::string& b) {
  auto parse = [](const std::string& s, long v[6]) {
    auto num = [&](size_t p, size_t n) { return std::strtol(s.substr(p, n).c_str(), nullptr, 10); };
    v[0] = num(0, 4); v[1] = num(4, 2); v[2] = num(6, 2); v[3] = num(9, 2); v[4] = num(11, 2); v[5] = num(13, 2);
  };
  long x[6], y[6];
  parse(a, x);
  parse(b, y);
  long j1 = julian_date(x[0], x[1], x[2]), j2 = julian_date(y[0], y[1], y[2]);
  return (j2 - j1) * 86400 + (y[3] * 3600 + y[4] * 60 + y[5]) - (x[3] * 3600 + x[4] * 60 + x[5]);
}

// compute_time_in_seconds: sfincs_spiderweb.f90:409-458.  "TIME = v unit since
// yyyy-mm-dd HH:MM:SS": v times the unit, minus (tref - that date), truncated to
// whole seconds, in the reference's real*4 / integer*8 steps.
static float meteo_time_seconds(const std::string& line, const std::string& trefstr) {
  const size_t j = line.find('='), jsince = line.find("since");
  size_t junit = std::string::npos;
  long ifac = 1;
  const char* units[4] = {"seconds", "minutes", "hours", "days"};
  const long facs[4] = {1, 60, 3600, 86400};
  for (int u = 0; u < 4 && junit == std::string::npos; u++) {
    junit = line.find(units[u]);
    ifac = facs[u];
  }
  if (j == std::string::npos || jsince == std::string::npos || junit == std::string::npos)
    throw std::runtime_error("oracle: bad TIME line in meteo file: " + line);
  const float tim = std::strtof(line.substr(j + 1, junit - j - 1).c_str(), nullptr);
  const std::string d = line.substr(jsince + 6, 19);  // yyyy-mm-dd HH:MM:SS
  const std::string datespw = d.substr(0, 4) + d.substr(5, 2) + d.substr(8, 2) + " " + d.substr(11, 2) +
                              d.substr(14, 2) + d.substr(17, 2);
  const long dts = time_difference(datespw, trefstr);
  const float v = tim * (float)ifac - (float)dts;
  return (float)(long long)v;
}

static std::vector<std::vector<double>> read_ascii_table(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<std::vector<double>> rows;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::vector<double> r;
    double x;
    while (is >> x) r.push_back(x);
    if (!r.empty()) rows.push_back(r);
  }
  return rows;
}

template <class X>
static std::vector<X> read_stream(const std::string& path, size_t n, size_t offset_bytes = 0) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  f.seekg((std::streamoff)offset_bytes);
  std::vector<X> out(n);
  f.read(reinterpret_cast<char*>(out.data()), (std::streamsize)(n * sizeof(X)));
  if (!f) throw std::runtime_error("short read " + path);
  return out;
}

// -------------------------------------------------------------------- model
template <class T, class TZ, class TV>
struct Model {
  std::string dir;
  std::string path(const std::string& f) const { return dir + "/" + f; }

  // --- inputs and switches (sfincs_input.f90:50-343, derived :347-745)
  int mmax, nmax;
  float dx, dy, x0, y0, rotation;
  std::string trefstr, tstartstr, tstopstr;
  float tspinup, alfa, theta, hmin_cfl, manning, manning_land, manning_sea, rghlevland, zini, qinf, dtmax,
      huthresh, huvmin, rhoa, rhow, latitude, pavbnd, gapres, advlim, slopelim, qinf_zmin, btfilter, btrelax,
      nuviscdim, wiggle_factor, wiggle_threshold, uvlim, uvmax, nuviscfac, dtmaxout, t0out = -999.0f;
  // max output (sfincs_lib.f90:430-445, sfincs_output.f90:197-230): the next
  // time, the count, and the fields as they were when last written
  double tmaxout = 1.0e9;
  long ntmaxout = 0;
  F1<T> zsmax_out, vmax_out, qmax_out, twet_out;
  F1<float> tzsmax_out;
  int bndtype, iadvection, baro, storevelmax, storefluxmax, storetwet, storetzsmax;
  std::string inputtype, advstr, qtrfile, depfile, zsinifile, rstfile, mskfile, indexfile, sbgfile, manningfile,
      bndfile, bzsfile, bcafile, bzifile, srcfile, disfile, wndfile, prcpfile, qinffile, scsfile, sefffile,
      psifile, f0file, infiltrationfile, inftype, thdfile, weirfile, drnfile;
  bool coriolis, viscosity, friction2d, advection_mask, wiggle_suppression, h73table, spinup_meteo;
  float t0, t1, g, pi, fcorio, twet_threshold;
  bool crsgeo = false, advection, thetasmoothing, subgrid, store_maximum_waterlevel, store_maximum_velocity,
       store_maximum_flux, store_twet, store_t_zsmax, use_quadtree, wind, precip, patmos, infiltration,
       use_qext, store_cumulative_precipitation = false;
  int advection_scheme = 1;

  // --- quadtree (sfincs_quadtree.F90:8-48)
  long qt_np;
  int qt_nlev;
  float qt_x0, qt_y0, qt_dx, qt_dy, qt_rot;
  int qt_nmax, qt_mmax;
  F1<int8_t> qt_level, qt_md, qt_mu, qt_nd, qt_nu;
  F1<int32_t> qt_md1, qt_md2, qt_mu1, qt_mu2, qt_nd1, qt_nd2, qt_nu1, qt_nu2, qt_n, qt_m, qt_nm_indices,
      qt_first, qt_last;
  F1<float> qt_dxr, qt_dyr, qt_zz;
  float qt_cosrot, qt_sinrot;

  // --- mesh (sfincs_data.f90)
  long np, npuv, ncuv;
  int nref;
  F1<int8_t> kcs, kcuv, kfuv, uv_flags_iref, uv_flags_type, uv_flags_dir, z_flags_iref, mask_adv;
  F1<int32_t> index_sfincs_in_quadtree, index_quadtree_in_sfincs, z_index_z_n, z_index_z_m, z_index_uv_md,
      z_index_uv_mu, z_index_uv_nd, z_index_uv_nu, z_index_uv_md1, z_index_uv_md2, z_index_uv_mu1, z_index_uv_mu2,
      z_index_uv_nd1, z_index_uv_nd2, z_index_uv_nu1, z_index_uv_nu2, uv_index_z_nm, uv_index_z_nmu,
      uv_index_u_nmd, uv_index_u_nmu, uv_index_u_ndm, uv_index_u_num, uv_index_v_ndm, uv_index_v_nm,
      uv_index_v_ndmu, uv_index_v_nmu, cuv_index_uv, cuv_index_uv1, cuv_index_uv2;
  F1<float> dxr, dyr, dxyr, z_xz, z_yz, dxrm, dxrinv, dxr2inv, dxrinvc, dyrm, dyrinv, dyr2inv, dyrinvc, cell_area,
      nuvisc;
  // geographic grids (sfincs_domain.f90:1403-1473): per uv point the inverse
  // width across it, per cell the width, area and Coriolis parameter
  F1<float> dxminv, dxm2inv, dxm, cell_area_m2, fcorio2d;
  float dtmin = 0.0f, cosrot, sinrot;
  float area_of(long nm) const { return crsgeo ? cell_area_m2(nm) : cell_area(z_flags_iref(nm)); }

  // --- bathymetry / subgrid
  F1<float> zb, zbuv, zbuvmx, gn2uv;
  int subgrid_nlevels = 0;
  F1<float> sg_z_zmin, sg_z_zmax, sg_z_volmax, sg_uv_zmin, sg_uv_zmax, sg_uv_navg_w, sg_uv_fnfit, sg_uv_havg_zmax,
      sg_uv_nrep_zmax;
  F2<float> sg_z_dep, sg_uv_havg, sg_uv_nrep, sg_uv_pwet;

  // --- boundaries
  long ngbnd = 0, nkcuv2 = 0, nbnd = 0, ntbnd = 0, itbndlast = 1;
  bool boundaries_in_mask = false, water_level_boundaries_in_mask = false, outflow_boundaries_in_mask = false,
       downstream_river_boundaries_in_mask = false, neumann_boundaries_in_mask = false;
  F1<int32_t> nmindbnd, index_kcuv2, nmbkcuv2, nmikcuv2, ibkcuv2, ind1_bnd_gbp, ind2_bnd_gbp, nmi_gbp;
  F1<int8_t> ibuvdir;
  F1<float> zsb, zsb0, uvmean, fac_bnd_gbp, x_bnd, y_bnd, t_bnd, zst_bnd;
  // downstream river boundaries (sfincs_boundaries.f90:217-270, 596-613, 878-902)
  long nbdr = 0;
  F1<float> x_bdr, y_bdr, dzs_bdr;
  F1<int32_t> index_zsi_bdr, index_bdr_gbp;
  std::string bdrfile;
  F2<float> zs_bnd;
  // astronomic constituents (sfincs_boundaries.f90:289-450; sfincs_data.f90:672-674)
  bool use_bcafile = true;
  long nr_tidal_components = 0;
  std::vector<double> tidal_component_frequency;      // [ic-1], rad/s
  std::vector<double> tidal_amp, tidal_phase;         // [(ib-1) * nc + ic-1]
  std::vector<std::string> tidal_component_names;

  // --- meteo, infiltration, sources
  long ntwnd = 0, itwndlast = 1, ntprcp = 0, itprcplast = 1;
  F1<float> twnd, wndmag, wnddir, tprcpt, tprcpv, cdval;
  F1<float> tauwu, tauwv, prcp, netprcp, qext, qinffield, qinfmap, cumprcp, cuminf;
  // gridded meteo on equidistant grids (ASCII amu/amv/amp/ampr, sfincs_meteo.f90:5-446, 802-1243):
  // the raw fields, the two fields of the current update window on the cells,
  // and the per-step values
  struct AmGrid {
    int nt = 0, nrows = 0, ncols = 0;
    float x_ll = 0, y_ll = 0, dx = 0, dy = 0;
    std::vector<float> times, v[2];  // v[q][((it - 1) * nrows + irow - 1) * ncols + icol - 1]
    float at(int q, int it, int irow, int icol) const {
      return v[q][((size_t)(it - 1) * nrows + (irow - 1)) * ncols + (icol - 1)];
    }
  };
  AmGrid amuv, amp, ampr;
  std::string amufile, amvfile, ampfile, amprfile;
  // spiderweb (sfincs_data.f90:686-762): polar records around the eye track
  struct SpwData {
    int nt = 0, nrows = 0, ncols = 0, nquant = 0;
    float radius = 0, drad = 0, dphi = 0;
    std::vector<float> times, xe, ye, wu, wv, pabs, prcp;  // [(it-1)*nrows*ncols + (irow-1)*ncols + icol-1]
    size_t at(int it, int irow, int icol) const {
      return ((size_t)(it - 1) * nrows + (irow - 1)) * ncols + (icol - 1);
    }
  };
  SpwData spw;
  std::string spwfile = "none", utmzone = "nil", z0lfile = "none";
  bool use_spw_precip = true, spw_precip = false;
  float spw_merge_frac = 0.5f, factor_spw_size = 1.0f;
  bool meteo3d = false, ampr_block = true;

  float dtwindupd = 1800.0f, twindupd = 0.0f, meteo_t0 = 0.0f, meteo_t1 = 0.0f, factor_wind = 1.0f,
        factor_pres = 1.0f, factor_prcp = 1.0f;
  F1<float> tauwu0, tauwu1, tauwv0, tauwv1, patm, patm0, patm1, prcp0, prcp1, patmb;
  // infiltration models with state (sfincs_infiltration.f90:8-600): curve number
  // with recovery (scs_*), Green-Ampt (GA_*), Horton (horton_*), recovery clock
  F1<float> scs_Se, scs_P1, scs_F1, scs_S1, ksfield, inf_kr, rain_T1, GA_head, GA_sigma, GA_sigma_max, GA_F, GA_Lu,
      horton_fc, horton_f0, horton_kd;
  F1<int> scs_rain;
  float sfacinf = 0.2f, horton_kr_kd = 10.0f;
  std::string smaxfile, sigmafile, ksfile, fcfile, kdfile;
  long nsrc = 0, ntsrc = 0, itsrclast = 1, ndrn = 0, nsrcdrn = 0;
  float structure_relax = 10.0f;
  F1<int8_t> drainage_type, drainage_status;
  F2<float> drainage_params;  // (ndrn, 6)
  F1<float> drainage_distance, drainage_fraction_open;
  F1<int32_t> nmindsrc;
  F1<float> tsrc, qtsrc;
  F2<float> qsrc;

  // --- structures (sfincs_data.f90: structure_*)
  long nrstructures = 0;
  F1<int32_t> structure_uv_index;
  F1<int8_t> structure_type;
  F1<float> structure_length;
  F2<float> structure_parameters;

  // --- hydro state
  F1<TZ> zs;
  F1<TV> z_volume;
  F1<T> q, q0, uv, uv0, zs0, zsderv, zsmax, vmax, qmax, twet;
  F1<float> t_zsmax;
  F1<T> x73;  // unused unless h73table (power7over3, sfincs_momentum.f90:787-820)

  // --- time loop
  double t;
  float dt, min_dt, dtavg;
  long nt = 0;
  int error = 0;

  // ================================================================ init
  void read_sfincs_input() {  // sfincs_input.f90:5-747 (hot-path keywords)
    InpFile in(path("sfincs.inp"));
    mmax = in.integer("mmax", 0);
    nmax = in.integer("nmax", 0);
    dx = in.real("dx", 0.0f);
    dy = in.real("dy", 0.0f);
    x0 = in.real("x0", 0.0f);
    y0 = in.real("y0", 0.0f);
    rotation = in.real("rotation", 0.0f);
    trefstr = in.str("tref", "none");
    tstartstr = in.str("tstart", "20000101 000000");
    tstopstr = in.str("tstop", "20000101 000000");
    tspinup = in.real("tspinup", 0.0f);
    dtmaxout = in.real("dtmaxout", 9999999.0f);
    t0out = in.real("t0out", -999.0f);
    alfa = in.real("alpha", 0.50f);
    theta = in.real("theta", 1.0f);
    hmin_cfl = in.real("hmin_cfl", 0.1f);
    manning = in.real("manning", 0.04f);
    manning_land = in.real("manning_land", -999.0f);
    manning_sea = in.real("manning_sea", -999.0f);
    rghlevland = in.real("rgh_lev_land", 0.0f);
    zini = in.real("zsini", 0.0f);
    qinf = in.real("qinf", 0.0f);
    dtmax = in.real("dtmax", 60.0f);
    huthresh = in.real("huthresh", 0.05f);
    huvmin = in.real("huvmin", 0.0f);
    rhoa = in.real("rhoa", 1.25f);
    rhow = in.real("rhow", 1024.0f);
    inputtype = in.str("inputformat", "bin");
    bndtype = in.integer("bndtype", 1);
    iadvection = in.integer("advection", 1);
    latitude = in.real("latitude", 0.0f);
    pavbnd = in.real("pavbnd", 0.0f);
    gapres = in.real("gapres", 101200.0f);
    baro = in.integer("baro", 1);
    advlim = in.real("advlim", 1.0f);
    slopelim = in.real("slopelim", 9999.9f);
    qinf_zmin = in.real("qinf_zmin", 0.0f);
    btfilter = in.real("btfilter", 60.0f);
    coriolis = in.logical("coriolis", true);
    nuviscdim = in.real("nuvisc", 0.01f);
    viscosity = in.logical("viscosity", false);
    spinup_meteo = in.integer("spinup_meteo", 0) != 0;
    amufile = in.str("amufile", "none");
    amvfile = in.str("amvfile", "none");
    ampfile = in.str("ampfile", "none");
    amprfile = in.str("amprfile", "none");
    spwfile = in.str("spwfile", "none");  // sfincs_input.f90:95-108, 203, 236, 247, 601-604
    utmzone = in.str("utmzone", "nil");
    z0lfile = in.str("z0lfile", "none");
    spw_merge_frac = in.real("spwmergefrac", 0.5f);
    use_spw_precip = in.integer("usespwprecip", 1) != 0;
    factor_spw_size = in.real("factor_spw_size", 1.0f);
    if (spwfile.substr(0, 4) != "none" && (utmzone != "nil" || z0lfile.substr(0, 4) != "none"))
      throw std::runtime_error("oracle: spiderweb reprojection and wind reduction are not restated");
    dtwindupd = in.real("dtwnd", 1800.0f);
    ampr_block = in.integer("amprblock", 1) != 0;
    factor_wind = in.real("factor_wind", 1.0f);
    factor_pres = in.real("factor_pres", 1.0f);
    factor_prcp = in.real("factor_prcp", 1.0f);
    if (in.real("waveage", -999.0f) > 0.0f || in.integer("radstr", 0) == 1)
      throw std::runtime_error("oracle: wave-age drag and radiation stresses are not restated");
    advstr = in.str("advection_scheme", "upw1");
    btrelax = in.real("btrelax", 3600.0f);
    wiggle_suppression = in.logical("wiggle_suppression", true);
    wiggle_factor = in.real("wiggle_factor", 0.1f);
    wiggle_threshold = in.real("wiggle_threshold", 0.1f);
    uvlim = in.real("uvlim", 10.0f);
    uvmax = in.real("uvmax", 1000.0f);
    friction2d = in.logical("friction2d", true);
    advection_mask = in.logical("advection_mask", true);
    nuviscfac = in.real("nuviscfac", 100.0f);
    h73table = in.logical("h73table", false);
    qtrfile = in.str("qtrfile", "none");
    depfile = in.str("depfile", "none");
    zsinifile = in.str("inifile", "none");
    rstfile = in.str("rstfile", "none");
    mskfile = in.str("mskfile", "none");
    indexfile = in.str("indexfile", "none");
    sbgfile = in.str("sbgfile", "none");
    manningfile = in.str("manningfile", "none");
    bndfile = in.str("bndfile", "none");
    bdrfile = in.str("bdrfile", "none");
    bzsfile = in.str("bzsfile", "none");
    bcafile = in.str("bcafile", "none");
    crsfile = in.str("crsfile", "none");
    rugfile = in.str("rugfile", "none");
    runup_gauge_depth = in.real("rugdepth", 0.05f);
    use_bcafile = in.logical("use_bcafile", true);
    bzifile = in.str("bzifile", "none");
    srcfile = in.str("srcfile", "none");
    disfile = in.str("disfile", "none");
    thdfile = in.str("thdfile", "none");
    weirfile = in.str("weirfile", "none");
    drnfile = in.str("drnfile", "none");
    structure_relax = in.real("structure_relax", 10.0f);
    wndfile = in.str("wndfile", "none");
    prcpfile = in.str("prcfile", "none");
    if (prcpfile.substr(0, 4) == "none") prcpfile = in.str("precipfile", "none");
    qinffile = in.str("qinffile", "none");
    scsfile = in.str("scsfile", "none");
    sefffile = in.str("sefffile", "none");
    psifile = in.str("psifile", "none");
    f0file = in.str("f0file", "none");
    smaxfile = in.str("smaxfile", "none");
    sigmafile = in.str("sigmafile", "none");
    ksfile = in.str("ksfile", "none");
    fcfile = in.str("fcfile", "none");
    kdfile = in.str("kdfile", "none");
    sfacinf = in.real("sfacinf", 0.2f);
    horton_kr_kd = in.real("horton_kr_kd", 10.0f);
    store_cumulative_precipitation = in.integer("storecumprcp", 0) == 1;
    infiltrationfile = in.str("infiltration_file", "none");
    inftype = in.str("infiltration_type", "none");
    storevelmax = in.integer("storevelmax", 0);
    storefluxmax = in.integer("storefluxmax", 0);
    storetwet = in.integer("storetwet", 0);
    storetzsmax = in.integer("storetzsmax", 0);
    twet_threshold = in.real("twet_threshold", 0.01f);
    int igeo = in.integer("crsgeo", 0);
    if (trefstr.substr(0, 4) == "none") trefstr = tstartstr;
    t0 = (float)(time_difference(trefstr, tstartstr) * 1.0);
    t1 = (float)(time_difference(trefstr, tstopstr) * 1.0);
    tspinup = t0 + tspinup;
    g = 9.81f;
    pi = 3.14159f;
    qinf = qinf / (float)(3600 * 1000);
    rotation = rotation * pi / 180.0f;
    cosrot = std::cos(rotation);
    sinrot = std::sin(rotation);
    fcorio = 0.0f;
    crsgeo = igeo != 0;  // sfincs_input.f90:399-421
    if (crsgeo && (weirfile.substr(0, 4) != "none" || drnfile.substr(0, 4) != "none" ||
                   spwfile.substr(0, 4) != "none"))
      throw std::runtime_error("oracle: weirs, drainage and spiderwebs on geographic grids are not restated");
    if (!crsgeo) {  // projected: Coriolis from the latitude, off near the equator
      fcorio = 2.0f * 7.2921e-05f * std::sin(latitude * pi / 180.0f);
      if (latitude < 0.01f && latitude > -0.01f) coriolis = false;
    }  // geographic: Coriolis per cell (fcorio2d), on unless the input turns it off
    if (t0out < -900.0f) t0out = t0;  // sfincs_input.f90:441-444
    t0out = std::max(t0out, t0);
    store_maximum_waterlevel = dtmaxout > 0.0f;
    store_maximum_velocity = storevelmax == 1 && dtmaxout > 0.0f;
    store_maximum_flux = storefluxmax == 1 && dtmaxout > 0.0f;
    store_twet = storetwet == 1;
    store_t_zsmax = storetzsmax == 1;
    subgrid = sbgfile.substr(0, 4) != "none";
    advection = iadvection > 0;
    thetasmoothing = theta < 0.9999f;
    if (advection) {
      advection_scheme = 1;
      if (advstr == "original") advection_scheme = 0;
    }
  }

  // initialize_processes: sfincs_domain.f90:59-140 (time-series meteo only)
  void initialize_processes() {
    use_quadtree = qtrfile.substr(0, 4) != "none";
    auto has = [](const std::string& f) { return f.substr(0, 4) != "none"; };
    wind = has(wndfile) || has(amufile) || has(spwfile);
    patmos = (has(ampfile) || has(spwfile)) && baro == 1;
    precip = has(prcpfile) || has(amprfile) || spw_precip;
    meteo3d = has(amufile) || has(amprfile) || has(ampfile) || has(spwfile);
  }

  // make_quadtree_from_indices: sfincs_quadtree.F90:445-669
  void make_quadtree_from_indices(long n_act, const std::vector<int32_t>& indices) {
    std::vector<int32_t> vm(n_act + 1), vn(n_act + 1), vnmu(n_act + 1, 0), vnmd(n_act + 1, 0), vnum(n_act + 1, 0),
        vndm(n_act + 1, 0);
    std::vector<int32_t> g((size_t)nmax * mmax, 0);
    auto G = [&](long n, long m) -> int32_t& { return g[(size_t)(m - 1) * nmax + (n - 1)]; };
    for (long nm = 1; nm <= n_act; nm++) {
      long m = (indices[nm - 1] - 1) / nmax + 1;
      long n = indices[nm - 1] - (m - 1) * nmax;
      vm[nm] = (int32_t)m;
      vn[nm] = (int32_t)n;
      G(n, m) = (int32_t)nm;
    }
    for (long nm = 1; nm <= n_act; nm++) {
      long m = vm[nm], n = vn[nm];
      if (m < mmax) vnmu[nm] = G(n, m + 1);
      if (m > 1) vnmd[nm] = G(n, m - 1);
      if (n < nmax) vnum[nm] = G(n + 1, m);
      if (n > 1) vndm[nm] = G(n - 1, m);
    }
    qt_np = n_act;
    qt_nlev = 1;
    qt_nmax = nmax;
    qt_mmax = mmax;
    qt_x0 = x0;
    qt_y0 = y0;
    qt_dx = dx;
    qt_dy = dy;
    qt_rot = rotation;
    qt_cosrot = std::cos(qt_rot);
    qt_sinrot = std::sin(qt_rot);
    qt_dxr.alloc(1);
    qt_dyr.alloc(1);
    qt_dxr(1) = dx;
    qt_dyr(1) = dy;
    qt_level.alloc(n_act, 1);
    qt_md.alloc(n_act); qt_mu.alloc(n_act); qt_nd.alloc(n_act); qt_nu.alloc(n_act);
    qt_md1.alloc(n_act); qt_md2.alloc(n_act); qt_mu1.alloc(n_act); qt_mu2.alloc(n_act);
    qt_nd1.alloc(n_act); qt_nd2.alloc(n_act); qt_nu1.alloc(n_act); qt_nu2.alloc(n_act);
    qt_n.alloc(n_act); qt_m.alloc(n_act);
    for (long ip = 1; ip <= n_act; ip++) {
      qt_md1(ip) = vnmd[ip];
      qt_mu1(ip) = vnmu[ip];
      qt_nd1(ip) = vndm[ip];
      qt_nu1(ip) = vnum[ip];
      qt_n(ip) = vn[ip];
      qt_m(ip) = vm[ip];
    }
    build_qt_search();
  }

  void build_qt_search() {  // sfincs_quadtree.F90:154-186, 637-667
    qt_nm_indices.alloc(qt_np);
    qt_first.alloc(qt_nlev);
    qt_last.alloc(qt_nlev);
    int ireflast = 0;
    for (long ip = 1; ip <= qt_np; ip++) {
      int iref = qt_level(ip);
      long nmx = (long)qt_nmax << (iref - 1);
      qt_nm_indices(ip) = (int32_t)((qt_m(ip) - 1) * nmx + qt_n(ip));
      if (iref > ireflast) {
        qt_first(iref) = (int32_t)ip;
        ireflast = iref;
      }
      qt_last(iref) = (int32_t)ip;
    }
  }

  // quadtree_read_file + quadtree_read_file_netcdf: sfincs_quadtree.F90:64-160, 295-440
  std::vector<int8_t> read_quadtree_netcdf() {
    if (qtrfile.find(".nc") == std::string::npos)
      throw std::runtime_error("oracle: only netCDF quadtree files are restated");
    nc3::File nc(path(qtrfile));
    qt_np = (long)nc.dim("mesh2d_nFaces");
    auto i32 = [&](const char* v, F1<int32_t>& a) {
      auto d = nc.read_double(v);
      a.alloc(qt_np);
      for (long i = 1; i <= qt_np; i++) a(i) = (int32_t)d[i - 1];
    };
    auto i8 = [&](const char* v, F1<int8_t>& a) {
      auto d = nc.read_double(v);
      a.alloc(qt_np);
      for (long i = 1; i <= qt_np; i++) a(i) = (int8_t)d[i - 1];
    };
    i32("n", qt_n);
    i32("m", qt_m);
    i8("level", qt_level);
    i8("md", qt_md); i32("md1", qt_md1); i32("md2", qt_md2);
    i8("mu", qt_mu); i32("mu1", qt_mu1); i32("mu2", qt_mu2);
    i8("nd", qt_nd); i32("nd1", qt_nd1); i32("nd2", qt_nd2);
    i8("nu", qt_nu); i32("nu1", qt_nu1); i32("nu2", qt_nu2);
    {
      auto z = nc.read_double("z");
      qt_zz.alloc(qt_np);
      for (long i = 1; i <= qt_np; i++) qt_zz(i) = (float)z[i - 1];
    }
    std::vector<int8_t> mskq((size_t)qt_np);
    {
      auto mk = nc.read_double("mask");
      for (long i = 0; i < qt_np; i++) mskq[(size_t)i] = (int8_t)mk[(size_t)i];
    }
    qt_x0 = (float)nc.att("x0");
    qt_y0 = (float)nc.att("y0");
    qt_dx = (float)nc.att("dx");
    qt_dy = (float)nc.att("dy");
    qt_rot = (float)nc.att("rotation");
    qt_nmax = (int)nc.att("nmax");
    qt_mmax = (int)nc.att("mmax");
    qt_nlev = (int)nc.att("nr_levels");
    const float pi = 3.141592653589793f;
    qt_rot = qt_rot * pi / 180.0f;
    qt_cosrot = std::cos(qt_rot);
    qt_sinrot = std::sin(qt_rot);
    qt_dxr.alloc(qt_nlev);
    qt_dyr.alloc(qt_nlev);
    for (int iref = 1; iref <= qt_nlev; iref++) {
      qt_dxr(iref) = qt_dx / (float)(1 << (iref - 1));
      qt_dyr(iref) = qt_dy / (float)(1 << (iref - 1));
    }
    for (long nm = 1; nm <= qt_np; nm++) {  // :118-126
      int iref = qt_level(nm);
      qt_nmax = std::max(qt_nmax, (int)((1.0f * (qt_n(nm) - 1) + 0.01f) / (float)(1 << (iref - 1))) + 1);
      qt_mmax = std::max(qt_mmax, (int)((1.0f * (qt_m(nm) - 1) + 0.01f) / (float)(1 << (iref - 1))) + 1);
    }
    build_qt_search();
    return mskq;
  }

  // initialize_mesh: sfincs_domain.f90:143-1586
  void initialize_mesh() {
    std::vector<int8_t> mskq;
    if (inputtype != "bin") throw std::runtime_error("oracle: only inputformat=bin is restated");
    if (use_quadtree) {
      mskq = read_quadtree_netcdf();  // :193-215 (netCDF quadtree: the mask comes with the file, :302-305)
      x0 = qt_x0;
      y0 = qt_y0;
      nmax = qt_nmax;
      mmax = qt_mmax;
      dx = qt_dx;
      dy = qt_dy;
    } else {
      auto head = read_stream<int32_t>(path(indexfile), 1);
      long n_act = head[0];
      auto idx = read_stream<int32_t>(path(indexfile), (size_t)n_act, 4);
      make_quadtree_from_indices(n_act, idx);
      mskq = read_stream<int8_t>(path(mskfile), (size_t)n_act);
    }
    rotation = qt_rot;
    nref = qt_nlev;
    // count and remap active points (:327-482)
    index_sfincs_in_quadtree.alloc(qt_np);
    np = 0;
    for (long ip = 1; ip <= qt_np; ip++)
      if (mskq[ip - 1] > 0) np++;
    kcs.alloc(np);
    index_quadtree_in_sfincs.alloc(np);
    z_flags_iref.alloc(np);
    F1<int8_t> z_flags_md, z_flags_mu, z_flags_nd, z_flags_nu;
    F1<int32_t> z_index_z_md1, z_index_z_md2, z_index_z_mu1, z_index_z_mu2, z_index_z_nd1, z_index_z_nd2,
        z_index_z_nu1, z_index_z_nu2, z_index_cuv_md, z_index_cuv_mu, z_index_cuv_nd, z_index_cuv_nu;
    z_flags_md.alloc(np); z_flags_mu.alloc(np); z_flags_nd.alloc(np); z_flags_nu.alloc(np);
    z_index_z_md1.alloc(np); z_index_z_md2.alloc(np); z_index_z_mu1.alloc(np); z_index_z_mu2.alloc(np);
    z_index_z_nd1.alloc(np); z_index_z_nd2.alloc(np); z_index_z_nu1.alloc(np); z_index_z_nu2.alloc(np);
    z_index_z_n.alloc(np); z_index_z_m.alloc(np);
    z_index_uv_md1.alloc(np); z_index_uv_md2.alloc(np); z_index_uv_mu1.alloc(np); z_index_uv_mu2.alloc(np);
    z_index_uv_nd1.alloc(np); z_index_uv_nd2.alloc(np); z_index_uv_nu1.alloc(np); z_index_uv_nu2.alloc(np);
    z_index_uv_md.alloc(np); z_index_uv_mu.alloc(np); z_index_uv_nd.alloc(np); z_index_uv_nu.alloc(np);
    z_index_cuv_md.alloc(np); z_index_cuv_mu.alloc(np); z_index_cuv_nd.alloc(np); z_index_cuv_nu.alloc(np);
    np = 0;
    for (long ip = 1; ip <= qt_np; ip++) {
      if (mskq[ip - 1] > 0) {
        np++;
        index_sfincs_in_quadtree(ip) = (int32_t)np;
        index_quadtree_in_sfincs(np) = (int32_t)ip;
      }
    }
    for (long ip = 1; ip <= np; ip++) {
      long iq = index_quadtree_in_sfincs(ip);
      kcs(ip) = mskq[iq - 1];
      z_flags_iref(ip) = qt_level(iq);
      z_index_z_n(ip) = qt_n(iq);
      z_index_z_m(ip) = qt_m(iq);
      z_flags_nu(ip) = qt_nu(iq);
      z_flags_nd(ip) = qt_nd(iq);
      z_flags_mu(ip) = qt_mu(iq);
      z_flags_md(ip) = qt_md(iq);
      if (qt_nu1(iq) > 0) z_index_z_nu1(ip) = index_sfincs_in_quadtree(qt_nu1(iq));
      if (qt_nu2(iq) > 0) z_index_z_nu2(ip) = index_sfincs_in_quadtree(qt_nu2(iq));
      if (qt_nd1(iq) > 0) z_index_z_nd1(ip) = index_sfincs_in_quadtree(qt_nd1(iq));
      if (qt_nd2(iq) > 0) z_index_z_nd2(ip) = index_sfincs_in_quadtree(qt_nd2(iq));
      if (qt_mu1(iq) > 0) z_index_z_mu1(ip) = index_sfincs_in_quadtree(qt_mu1(iq));
      if (qt_mu2(iq) > 0) z_index_z_mu2(ip) = index_sfincs_in_quadtree(qt_mu2(iq));
      if (qt_md1(iq) > 0) z_index_z_md1(ip) = index_sfincs_in_quadtree(qt_md1(iq));
      if (qt_md2(iq) > 0) z_index_z_md2(ip) = index_sfincs_in_quadtree(qt_md2(iq));
    }
    // count u and v points (:486-533)
    long npu = 0, npv = 0;
    for (long nm = 1; nm <= np; nm++) {
      if (z_flags_mu(nm) < 1) {
        if (z_index_z_mu1(nm) > 0) npu++;
      } else {
        if (z_index_z_mu1(nm) > 0) npu++;
        if (z_index_z_mu2(nm) > 0) npu++;
      }
      if (z_flags_nu(nm) < 1) {
        if (z_index_z_nu1(nm) > 0) npv++;
      } else {
        if (z_index_z_nu1(nm) > 0) npv++;
        if (z_index_z_nu2(nm) > 0) npv++;
      }
    }
    npuv = npu + npv;
    ncuv = 0;
    if (qt_nlev > 1) {  // :537-596
      for (long nm = 1; nm <= np; nm++) {
        if (z_flags_md(nm) == 1 && (z_index_z_md1(nm) > 0 || z_index_z_md2(nm) > 0)) ncuv++;
        if (z_flags_mu(nm) == 1 && (z_index_z_mu1(nm) > 0 || z_index_z_mu2(nm) > 0)) ncuv++;
        if (z_flags_nd(nm) == 1 && (z_index_z_nd1(nm) > 0 || z_index_z_nd2(nm) > 0)) ncuv++;
        if (z_flags_nu(nm) == 1 && (z_index_z_nu1(nm) > 0 || z_index_z_nu2(nm) > 0)) ncuv++;
      }
    }
    long npuvtotal = npuv + ncuv;
    z_index_uv_md.fill((int32_t)(npuvtotal + 1));
    z_index_uv_mu.fill((int32_t)(npuvtotal + 1));
    z_index_uv_nd.fill((int32_t)(npuvtotal + 1));
    z_index_uv_nu.fill((int32_t)(npuvtotal + 1));
    cuv_index_uv.alloc(ncuv);
    cuv_index_uv1.alloc(ncuv, (int32_t)(npuvtotal + 1));
    cuv_index_uv2.alloc(ncuv, (int32_t)(npuvtotal + 1));
    long irefuv = 0;  // :618-678
    for (long nm = 1; nm <= np; nm++) {
      if (z_flags_md(nm) == 1 && (z_index_z_md1(nm) > 0 || z_index_z_md2(nm) > 0)) {
        irefuv++;
        cuv_index_uv(irefuv) = (int32_t)(npuv + irefuv);
        z_index_cuv_md(nm) = (int32_t)irefuv;
      }
      if (z_flags_mu(nm) == 1 && (z_index_z_mu1(nm) > 0 || z_index_z_mu2(nm) > 0)) {
        irefuv++;
        cuv_index_uv(irefuv) = (int32_t)(npuv + irefuv);
        z_index_cuv_mu(nm) = (int32_t)irefuv;
      }
      if (z_flags_nd(nm) == 1 && (z_index_z_nd1(nm) > 0 || z_index_z_nd2(nm) > 0)) {
        irefuv++;
        cuv_index_uv(irefuv) = (int32_t)(npuv + irefuv);
        z_index_cuv_nd(nm) = (int32_t)irefuv;
      }
      if (z_flags_nu(nm) == 1 && (z_index_z_nu1(nm) > 0 || z_index_z_nu2(nm) > 0)) {
        irefuv++;
        cuv_index_uv(irefuv) = (int32_t)(npuv + irefuv);
        z_index_cuv_nu(nm) = (int32_t)irefuv;
      }
    }
    kcuv.alloc(npuv + ncuv + 1);
    uv_index_z_nm.alloc(npuv);
    uv_index_z_nmu.alloc(npuv);
    uv_flags_iref.alloc(npuv);
    uv_flags_dir.alloc(npuv);
    uv_flags_type.alloc(npuv);
    bool need8 = advection || coriolis || viscosity || thetasmoothing || friction2d;
    if (need8) {
      uv_index_u_nmd.alloc(npuv); uv_index_u_nmu.alloc(npuv); uv_index_u_num.alloc(npuv);
      uv_index_u_ndm.alloc(npuv); uv_index_v_ndm.alloc(npuv); uv_index_v_nm.alloc(npuv);
      uv_index_v_ndmu.alloc(npuv); uv_index_v_nmu.alloc(npuv);
    }
    long ip = 0;  // uv enumeration :721-1003
    for (long nm = 1; nm <= np; nm++) {
      long nmu, num, icuv;
      if (z_flags_mu(nm) == 0) {
        if (z_index_z_mu1(nm) > 0) {
          ip++;
          nmu = z_index_z_mu1(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)nmu;
          z_index_uv_mu(nm) = (int32_t)ip;
          z_index_uv_md(nmu) = (int32_t)ip;
          z_index_uv_mu1(nm) = (int32_t)ip;
          z_index_uv_md1(nmu) = (int32_t)ip;
          uv_flags_iref(ip) = z_flags_iref(nm);
          uv_flags_dir(ip) = 0;
          uv_flags_type(ip) = 0;
        }
      } else if (z_flags_mu(nm) == -1) {
        if (z_index_z_mu1(nm) > 0) {
          ip++;
          nmu = z_index_z_mu1(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)nmu;
          z_index_uv_mu(nm) = (int32_t)ip;
          z_index_uv_mu1(nm) = (int32_t)ip;
          icuv = z_index_cuv_md(nmu);
          if (z_index_z_md1(z_index_z_mu1(nm)) == nm) {
            cuv_index_uv1(icuv) = (int32_t)ip;
            z_index_uv_md1(nmu) = (int32_t)ip;
          } else {
            cuv_index_uv2(icuv) = (int32_t)ip;
            z_index_uv_md2(nmu) = (int32_t)ip;
          }
          z_index_uv_md(nmu) = cuv_index_uv(icuv);
          uv_flags_iref(ip) = z_flags_iref(nm);
          uv_flags_dir(ip) = 0;
          uv_flags_type(ip) = -1;
        }
      } else {
        if (z_index_z_mu1(nm) > 0) {
          ip++;
          nmu = z_index_z_mu1(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)nmu;
          z_index_uv_mu1(nm) = (int32_t)ip;
          z_index_uv_md(nmu) = (int32_t)ip;
          z_index_uv_md1(nmu) = (int32_t)ip;
          icuv = z_index_cuv_mu(nm);
          z_index_uv_mu(nm) = cuv_index_uv(icuv);
          cuv_index_uv1(icuv) = (int32_t)ip;
          uv_flags_iref(ip) = (int8_t)(z_flags_iref(nm) + 1);
          uv_flags_dir(ip) = 0;
          uv_flags_type(ip) = 1;
        }
        if (z_index_z_mu2(nm) > 0) {
          ip++;
          nmu = z_index_z_mu2(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)nmu;
          z_index_uv_mu2(nm) = (int32_t)ip;
          z_index_uv_md(nmu) = (int32_t)ip;
          z_index_uv_md1(nmu) = (int32_t)ip;
          icuv = z_index_cuv_mu(nm);
          z_index_uv_mu(nm) = cuv_index_uv(icuv);
          cuv_index_uv2(icuv) = (int32_t)ip;
          uv_flags_iref(ip) = (int8_t)(z_flags_iref(nm) + 1);
          uv_flags_dir(ip) = 0;
          uv_flags_type(ip) = 1;
        }
      }
      if (z_flags_nu(nm) == 0) {
        if (z_index_z_nu1(nm) > 0) {
          ip++;
          num = z_index_z_nu1(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)num;
          z_index_uv_nu(nm) = (int32_t)ip;
          z_index_uv_nd(num) = (int32_t)ip;
          z_index_uv_nu1(nm) = (int32_t)ip;
          z_index_uv_nd1(num) = (int32_t)ip;
          uv_flags_iref(ip) = z_flags_iref(nm);
          uv_flags_dir(ip) = 1;
          uv_flags_type(ip) = 0;
        }
      } else if (z_flags_nu(nm) == -1) {
        if (z_index_z_nu1(nm) > 0) {
          ip++;
          num = z_index_z_nu1(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)num;
          z_index_uv_nu(nm) = (int32_t)ip;
          z_index_uv_nu1(nm) = (int32_t)ip;
          icuv = z_index_cuv_nd(num);
          if (z_index_z_nd1(z_index_z_nu1(nm)) == nm) {
            cuv_index_uv1(icuv) = (int32_t)ip;
            z_index_uv_nd1(num) = (int32_t)ip;
          } else {
            cuv_index_uv2(icuv) = (int32_t)ip;
            z_index_uv_nd2(num) = (int32_t)ip;
          }
          z_index_uv_nd(num) = cuv_index_uv(icuv);
          uv_flags_iref(ip) = z_flags_iref(nm);
          uv_flags_dir(ip) = 1;
          uv_flags_type(ip) = -1;
        }
      } else {
        if (z_index_z_nu1(nm) > 0) {
          ip++;
          num = z_index_z_nu1(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)num;
          z_index_uv_nd(num) = (int32_t)ip;
          z_index_uv_nu1(nm) = (int32_t)ip;
          z_index_uv_nd1(num) = (int32_t)ip;
          icuv = z_index_cuv_nu(nm);
          z_index_uv_nu(nm) = cuv_index_uv(icuv);
          cuv_index_uv1(icuv) = (int32_t)ip;
          uv_flags_iref(ip) = (int8_t)(z_flags_iref(nm) + 1);
          uv_flags_dir(ip) = 1;
          uv_flags_type(ip) = 1;
        }
        if (z_index_z_nu2(nm) > 0) {
          ip++;
          num = z_index_z_nu2(nm);
          uv_index_z_nm(ip) = (int32_t)nm;
          uv_index_z_nmu(ip) = (int32_t)num;
          z_index_uv_nd(num) = (int32_t)ip;
          z_index_uv_nu2(nm) = (int32_t)ip;
          z_index_uv_nd1(num) = (int32_t)ip;
          icuv = z_index_cuv_nu(nm);
          z_index_uv_nu(nm) = cuv_index_uv(icuv);
          cuv_index_uv2(icuv) = (int32_t)ip;
          uv_flags_iref(ip) = (int8_t)(z_flags_iref(nm) + 1);
          uv_flags_dir(ip) = 1;
          uv_flags_type(ip) = 1;
        }
      }
    }
    if (need8) {  // 8 uv neighbours :1007-1261
      for (long ip2 = 1; ip2 <= npuv; ip2++) {
        long nm = uv_index_z_nm(ip2);
        if (uv_flags_dir(ip2) == 0) {
          long nmu = uv_index_z_nmu(ip2);
          uv_index_u_nmd(ip2) = z_index_uv_md(nm);
          uv_index_u_nmu(ip2) = z_index_uv_mu(nmu);
          if (z_flags_nd(nm) > -1) {
            long ndm = z_index_z_nd1(nm);
            if (ndm > 0) uv_index_u_ndm(ip2) = z_index_uv_mu(ndm);
          } else {
            long ndm = z_index_z_nd2(nm);
            if (ndm > 0) {
              if (z_flags_mu(ndm) == 0) {
                uv_index_u_ndm(ip2) = z_index_uv_mu(ndm);
              } else {
                long ndmu = z_index_z_mu1(ndm);
                if (ndmu > 0) uv_index_u_ndm(ip2) = z_index_uv_md(ndmu);
              }
            }
          }
          if (z_flags_nu(nm) > -1) {
            long num = z_index_z_nu1(nm);
            if (num > 0) uv_index_u_num(ip2) = z_index_uv_mu(num);
          } else {
            long num = z_index_z_nu2(nm);
            if (num > 0) {
              if (z_flags_mu(num) == 0) {
                uv_index_u_num(ip2) = z_index_uv_mu(num);
              } else {
                long numu = z_index_z_mu1(num);
                if (numu > 0) uv_index_u_num(ip2) = z_index_uv_md(numu);
              }
            }
          }
          uv_index_v_nm(ip2) = z_index_uv_nu(nm);
          uv_index_v_ndm(ip2) = z_index_uv_nd(nm);
          uv_index_v_nmu(ip2) = z_index_uv_nu(nmu);
          uv_index_v_ndmu(ip2) = z_index_uv_nd(nmu);
        } else {
          long num = uv_index_z_nmu(ip2);
          uv_index_u_nmd(ip2) = z_index_uv_nd(nm);
          uv_index_u_nmu(ip2) = z_index_uv_nu(num);
          if (z_flags_md(nm) > -1) {
            long nmd = z_index_z_md1(nm);
            if (nmd > 0) uv_index_u_ndm(ip2) = z_index_uv_nu(nmd);
          } else {
            long nmd = z_index_z_md2(nm);
            if (nmd > 0) {
              if (z_flags_nu(nmd) == 0) {
                uv_index_u_ndm(ip2) = z_index_uv_nu(nmd);
              } else {
                long nmdu = z_index_z_nu1(nmd);
                if (nmdu > 0) uv_index_u_ndm(ip2) = z_index_uv_nd(nmdu);
              }
            }
          }
          if (z_flags_mu(nm) > -1) {
            long nmu = z_index_z_mu1(nm);
            if (nmu > 0) uv_index_u_num(ip2) = z_index_uv_nu(nmu);
          } else {
            long nmu = z_index_z_mu2(nm);
            if (nmu > 0) {
              if (z_flags_nu(nmu) == 0) {
                uv_index_u_num(ip2) = z_index_uv_nu(nmu);
              } else {
                long numu = z_index_z_nu1(nmu);
                if (numu > 0) uv_index_u_num(ip2) = z_index_uv_nd(numu);
              }
            }
          }
          uv_index_v_nm(ip2) = z_index_uv_mu(nm);
          uv_index_v_ndm(ip2) = z_index_uv_md(nm);
          uv_index_v_nmu(ip2) = z_index_uv_mu(num);
          uv_index_v_ndmu(ip2) = z_index_uv_md(num);
        }
        if (uv_index_u_nmd(ip2) == 0) uv_index_u_nmd(ip2) = (int32_t)ip2;
        if (uv_index_u_nmu(ip2) == 0) uv_index_u_nmu(ip2) = (int32_t)ip2;
        if (uv_index_u_ndm(ip2) == 0) uv_index_u_ndm(ip2) = (int32_t)ip2;
        if (uv_index_u_num(ip2) == 0) uv_index_u_num(ip2) = (int32_t)ip2;
        if (uv_index_v_ndm(ip2) == 0) uv_index_v_ndm(ip2) = (int32_t)(npuvtotal + 1);
        if (uv_index_v_ndmu(ip2) == 0) uv_index_v_ndmu(ip2) = (int32_t)(npuvtotal + 1);
        if (uv_index_v_nm(ip2) == 0) uv_index_v_nm(ip2) = (int32_t)(npuvtotal + 1);
        if (uv_index_v_nmu(ip2) == 0) uv_index_v_nmu(ip2) = (int32_t)(npuvtotal + 1);
      }
    }
    // geometry :1369-1541 (projected)
    dxr.alloc(nref); dyr.alloc(nref); dxyr.alloc(nref);
    for (int iref = 1; iref <= nref; iref++) {
      dxr(iref) = dx / (float)(1 << (iref - 1));
      dyr(iref) = dy / (float)(1 << (iref - 1));
      dxyr(iref) = std::min(dxr(iref), dyr(iref));
    }
    z_xz.alloc(np);
    z_yz.alloc(np);
    for (long nm = 1; nm <= np; nm++) {
      float n = (float)z_index_z_n(nm), m = (float)z_index_z_m(nm);
      int iref = z_flags_iref(nm);
      z_xz(nm) = x0 + cosrot * (1.0f * (m - 0.5f)) * dxr(iref) - sinrot * (1.0f * (n - 0.5f)) * dyr(iref);
      z_yz(nm) = y0 + sinrot * (1.0f * (m - 0.5f)) * dxr(iref) + cosrot * (1.0f * (n - 0.5f)) * dyr(iref);
    }
    float dxymin = 1.0e6f;
    dxrm.alloc(nref); dxrinv.alloc(nref); dxr2inv.alloc(nref); dxrinvc.alloc(nref);
    dyrm.alloc(nref); dyrinv.alloc(nref); dyr2inv.alloc(nref); dyrinvc.alloc(nref);
    cell_area.alloc(nref);
    if (crsgeo) {  // dxr, dyr in degrees (:1403-1473); no dtmax limit from the spacing, no dtmin
      dxminv.alloc(npuv);
      dxm2inv.alloc(npuv);
      dxm.alloc(np);
      cell_area_m2.alloc(np);
      fcorio2d.alloc(np);
      for (long ip = 1; ip <= npuv; ip++) {
        const int iref = use_quadtree ? uv_flags_iref(ip) : 1;
        const long nm = uv_index_z_nm(ip);
        dxminv(ip) = 1.0f / (dxr(iref) * 111111.1f * std::cos(z_yz(nm) * pi / 180.0f));
        dxm2inv(ip) = dxminv(ip) * dxminv(ip);
      }
      for (int iref = 1; iref <= nref; iref++) {
        dyrm(iref) = 111111.1f * dyr(iref);
        dyrinv(iref) = 1.0f / dyrm(iref);
        dyr2inv(iref) = dyrinv(iref) * dyrinv(iref);
        if (iref > 1) dyrinvc(iref) = 1.0f / (3.0f * dyrm(iref) / 2.0f);
      }
      for (long nm = 1; nm <= np; nm++) {
        const int iref = z_flags_iref(nm);
        dxm(nm) = dxr(iref) * 111111.1f * std::cos(z_yz(nm) * pi / 180.0f);
        cell_area_m2(nm) = dxm(nm) * dyrm(iref);
      }
      if (coriolis)
        for (long nm = 1; nm <= np; nm++) fcorio2d(nm) = 2.0f * 7.2921e-05f * std::sin(z_yz(nm) * pi / 180.0f);
      nuvisc.alloc(nref);
      if (viscosity)  // :1549-1559
        for (int iref = 1; iref <= nref; iref++) nuvisc(iref) = std::max(nuviscdim * dxyr(iref) / 0.00001f, 0.0f);
      return;
    }
    for (int iref = 1; iref <= nref; iref++) {
      dxrm(iref) = dxr(iref);
      dxrinv(iref) = 1.0f / dxrm(iref);
      dxr2inv(iref) = dxrinv(iref) * dxrinv(iref);
      dyrm(iref) = dyr(iref);
      dyrinv(iref) = 1.0f / dyrm(iref);
      dyr2inv(iref) = dyrinv(iref) * dyrinv(iref);
      cell_area(iref) = dxrm(iref) * dyrm(iref);
      if (iref > 1) {
        dxrinvc(iref) = 1.0f / (3.0f * dxrm(iref) / 2.0f);
        dyrinvc(iref) = 1.0f / (3.0f * dyrm(iref) / 2.0f);
      }
      dxymin = std::min(dxymin, dxr(iref));
      dxymin = std::min(dxymin, dyr(iref));
    }
    dtmax = std::min(dtmax, alfa * dxymin / (std::sqrt(9.81f * hmin_cfl)));
    dtmin = alfa * dxymin / (1.25f * std::fabs(uvmax));
    nuvisc.alloc(nref);
    if (viscosity)
      for (int iref = 1; iref <= nref; iref++) nuvisc(iref) = std::max(nuviscdim * dxyr(iref), 0.0f);
  }

  // initialize_bathymetry: sfincs_domain.f90:1588-1744
  void initialize_bathymetry() {
    if (!subgrid) {
      zb.alloc(np);
      zbuv.alloc(npuv);
      zbuvmx.alloc(npuv);
      if (use_quadtree && depfile.substr(0, 4) == "none") {  // :1618-1638
        for (long i = 1; i <= np; i++) zb(i) = qt_zz(index_quadtree_in_sfincs(i));
      } else {
        auto d = read_stream<float>(path(depfile), (size_t)np);
        for (long i = 1; i <= np; i++) zb(i) = d[i - 1];
      }
      for (long ip = 1; ip <= npuv; ip++) {
        long nm = uv_index_z_nm(ip), nmu = uv_index_z_nmu(ip);
        if (uv_flags_type(ip) == 0)
          zbuv(ip) = 0.5f * (zb(nm) + zb(nmu));
        else if (uv_flags_type(ip) == -1)
          zbuv(ip) = 0.3333f * zb(nm) + 0.6667f * zb(nmu);
        else
          zbuv(ip) = 0.6667f * zb(nm) + 0.3333f * zb(nmu);
        zbuvmx(ip) = std::max(zb(nm), zb(nmu)) + huthresh;
      }
    } else {
      read_subgrid_file_netcdf();
    }
  }

  // read_subgrid_file / read_subgrid_file_netcdf: sfincs_subgrid.F90:20-455
  void read_subgrid_file_netcdf() {
    huthresh = 0.0f;  // :40
    nc3::File nc(path(sbgfile));
    subgrid_nlevels = (int)nc.dim("levels");
    long L = subgrid_nlevels;
    auto zmin = nc.read_float("z_zmin"), zmax = nc.read_float("z_zmax"), volmax = nc.read_float("z_volmax"),
         zlev = nc.read_float("z_level"), uzmin = nc.read_float("uv_zmin"), uzmax = nc.read_float("uv_zmax"),
         uffit = nc.read_float("uv_ffit"), unavg = nc.read_float("uv_navg"), uhavg = nc.read_float("uv_havg"),
         unrep = nc.read_float("uv_nrep"), upwet = nc.read_float("uv_pwet");
    // file index (0-based) of every active cell and uv point: identity on a
    // regular grid (:246-270); on a quadtree the file covers every quadtree
    // point and its right/upper faces (:166-245)
    std::vector<long> zi((size_t)np), ui((size_t)npuv);
    if (use_quadtree) {
      long npuvq = 0, npuvs = 0;
      for (long ip = 1; ip <= qt_np; ip++) {
        long nm = index_sfincs_in_quadtree(ip);
        if (nm > 0) zi[(size_t)nm - 1] = ip - 1;
        auto face = [&](int32_t nb, const F1<int32_t>& zuv) {
          if (nb > 0) {
            npuvq++;
            if (nm > 0 && zuv(nm) > 0) {
              if (npuvs >= npuv) throw std::runtime_error("oracle: subgrid file faces do not match the mesh");
              ui[(size_t)npuvs++] = npuvq - 1;
            }
          }
        };
        if (qt_mu(ip) < 1) {
          face(qt_mu1(ip), z_index_uv_mu1);
        } else {
          face(qt_mu1(ip), z_index_uv_mu1);
          face(qt_mu2(ip), z_index_uv_mu2);
        }
        if (qt_nu(ip) < 1) {
          face(qt_nu1(ip), z_index_uv_nu1);
        } else {
          face(qt_nu1(ip), z_index_uv_nu1);
          face(qt_nu2(ip), z_index_uv_nu2);
        }
      }
      if ((long)zmin.size() != qt_np || (long)uzmin.size() != npuvq || npuvs != npuv)
        throw std::runtime_error("oracle: subgrid file does not match the quadtree mesh");
    } else {
      if ((long)zmin.size() != np || (long)uzmin.size() != npuv)
        throw std::runtime_error("oracle: subgrid file does not match the mesh");
      for (long i = 0; i < np; i++) zi[(size_t)i] = i;
      for (long i = 0; i < npuv; i++) ui[(size_t)i] = i;
    }
    sg_z_zmin.alloc(np); sg_z_zmax.alloc(np); sg_z_volmax.alloc(np); sg_z_dep.alloc(L, np);
    sg_uv_zmin.alloc(npuv); sg_uv_zmax.alloc(npuv); sg_uv_navg_w.alloc(npuv); sg_uv_fnfit.alloc(npuv);
    sg_uv_havg.alloc(L, npuv); sg_uv_nrep.alloc(L, npuv); sg_uv_pwet.alloc(L, npuv);
    sg_uv_havg_zmax.alloc(npuv); sg_uv_nrep_zmax.alloc(npuv);
    for (long ip = 1; ip <= np; ip++) {
      const long f = zi[(size_t)ip - 1];
      sg_z_zmin(ip) = zmin[f];
      sg_z_zmax(ip) = zmax[f];
      sg_z_volmax(ip) = volmax[f];
      for (long k = 1; k <= L; k++) sg_z_dep(k, ip) = zlev[f * L + (k - 1)];
    }
    for (long ip = 1; ip <= npuv; ip++) {
      const long f = ui[(size_t)ip - 1];
      sg_uv_zmin(ip) = uzmin[f];
      sg_uv_zmax(ip) = uzmax[f];
      sg_uv_zmax(ip) = std::max(sg_uv_zmax(ip), sg_uv_zmin(ip) + 0.01f);
      sg_uv_fnfit(ip) = uffit[f];
      float nv = std::max(unavg[f], 0.0001f);
      sg_uv_navg_w(ip) = g * (nv * nv);
      for (long k = 1; k <= L; k++) {
        sg_uv_havg(k, ip) = uhavg[f * L + (k - 1)];
        float nr = std::max(unrep[f * L + (k - 1)], 0.0001f);
        sg_uv_nrep(k, ip) = g * (nr * nr);
        sg_uv_pwet(k, ip) = upwet[f * L + (k - 1)];
      }
    }
    for (long ip = 1; ip <= npuv; ip++) {  // :364-388
      long nm = uv_index_z_nm(ip), nmu = uv_index_z_nmu(ip);
      if (sg_z_zmin(nm) > sg_uv_zmin(ip)) {
        sg_uv_zmin(ip) = std::max(sg_uv_zmin(ip), sg_z_zmin(nm));
        sg_uv_zmax(ip) = std::max(sg_uv_zmax(ip), sg_uv_zmin(ip) + 0.01f);
      }
      if (sg_z_zmin(nmu) > sg_uv_zmin(ip)) {
        sg_uv_zmin(ip) = std::max(sg_uv_zmin(ip), sg_z_zmin(nmu));
        sg_uv_zmax(ip) = std::max(sg_uv_zmax(ip), sg_uv_zmin(ip) + 0.01f);
      }
    }
    for (long nm = 1; nm <= np; nm++)  // :400-411
      if (sg_z_zmax(nm) - sg_z_zmin(nm) <= 0.0f) sg_z_zmax(nm) = sg_z_zmax(nm) + 0.01f;
    for (long ip = 1; ip <= npuv; ip++)  // :421-433
      if (sg_uv_zmax(ip) - sg_uv_zmin(ip) < 1.0e-7f) sg_uv_zmax(ip) = sg_uv_zmax(ip) + 0.01f;
    for (long ip = 1; ip <= npuv; ip++) {  // :443-446
      sg_uv_havg_zmax(ip) = sg_uv_havg(L, ip) - sg_uv_zmax(ip);
      sg_uv_nrep_zmax(ip) = sg_uv_nrep(L, ip);
    }
  }

  // initialize_boundaries: sfincs_domain.f90:1765-1958
  void initialize_boundaries() {
    ngbnd = 0;
    for (long nm = 1; nm <= np; nm++) {
      int k = kcs(nm);
      if (k == 2 || k == 3 || k == 5 || k == 6) {
        boundaries_in_mask = true;
        ngbnd++;
        if (k == 2) water_level_boundaries_in_mask = true;
        if (k == 3) outflow_boundaries_in_mask = true;
        if (k == 5) downstream_river_boundaries_in_mask = true;
        if (k == 6) neumann_boundaries_in_mask = true;
      }
    }
    nmindbnd.alloc(ngbnd);
    zsb.alloc(ngbnd);
    zsb0.alloc(ngbnd);
    ngbnd = 0;
    for (long nm = 1; nm <= np; nm++) {
      int k = kcs(nm);
      if (k == 2 || k == 3 || k == 5 || k == 6) nmindbnd(++ngbnd) = (int32_t)nm;
    }
    nkcuv2 = 0;
    kcuv.fill(0);
    for (long ip = 1; ip <= npuv; ip++) {
      int a = kcs(uv_index_z_nm(ip)), b = kcs(uv_index_z_nmu(ip));
      if (a > 1 && b > 1)
        kcuv(ip) = 0;
      else if (a * b == 0)
        kcuv(ip) = 0;
      else if ((a == 1 && b == 2) || (a == 2 && b == 1)) {
        kcuv(ip) = 2;
        nkcuv2++;
      } else if ((a == 1 && b == 3) || (a == 3 && b == 1)) {
        kcuv(ip) = 2;
        nkcuv2++;
      } else if ((a == 1 && b == 5) || (a == 5 && b == 1)) {
        kcuv(ip) = 2;
        nkcuv2++;
      } else if ((a == 1 && b == 6) || (a == 6 && b == 1)) {
        kcuv(ip) = 6;
        nkcuv2++;
      } else
        kcuv(ip) = 1;
    }
    index_kcuv2.alloc(nkcuv2); nmbkcuv2.alloc(nkcuv2); nmikcuv2.alloc(nkcuv2);
    ibuvdir.alloc(nkcuv2); uvmean.alloc(nkcuv2); ibkcuv2.alloc(nkcuv2);
    long ik = 0;
    for (long ip = 1; ip <= npuv; ip++) {
      if (kcuv(ip) == 2 || kcuv(ip) == 6) {
        ik++;
        index_kcuv2(ik) = (int32_t)ip;
        long nm = uv_index_z_nm(ip), nmu = uv_index_z_nmu(ip);
        if (kcs(nm) == 1) {
          nmbkcuv2(ik) = (int32_t)nmu;
          nmikcuv2(ik) = (int32_t)nm;
          ibuvdir(ik) = -1;
        } else {
          nmbkcuv2(ik) = (int32_t)nm;
          nmikcuv2(ik) = (int32_t)nmu;
          ibuvdir(ik) = 1;
        }
        for (long ib = 1; ib <= ngbnd; ib++) {
          if (nmindbnd(ib) == nmbkcuv2(ik)) {
            ibkcuv2(ik) = (int32_t)ib;
            if (kcs(nmindbnd(ib)) == 3) {
              zsb0(ib) = subgrid ? sg_z_zmin(nmindbnd(ib)) : zb(nmindbnd(ib));
              zsb(ib) = zsb0(ib);
            }
            break;
          }
        }
      }
    }
  }

  // initialize_roughness: sfincs_domain.f90:1960-2061
  void initialize_roughness() {
    if (subgrid) return;
    gn2uv.alloc(npuv, 9.81f * 0.02f * 0.02f);
    if (manningfile.substr(0, 4) != "none") {
      auto r = read_stream<float>(path(manningfile), (size_t)np);
      for (long ip = 1; ip <= npuv; ip++) {
        long nm = uv_index_z_nm(ip), nmu = uv_index_z_nmu(ip);
        if (kcuv(ip) > 0) {
          float a = 0.5f * (r[nm - 1] + r[nmu - 1]);
          gn2uv(ip) = 9.81f * (a * a);
        }
      }
    } else {
      float gn2land = manning_land < 0.0f ? 9.81f * (manning * manning) : 9.81f * (manning_land * manning_land);
      float gn2sea = manning_sea < 0.0f ? 9.81f * (manning * manning) : 9.81f * (manning_sea * manning_sea);
      for (long ip = 1; ip <= npuv; ip++)
        if (kcuv(ip) > 0) gn2uv(ip) = zbuv(ip) > rghlevland ? gn2land : gn2sea;
    }
  }

  // initialize_infiltration: sfincs_infiltration.f90:8-606 (con and c2d)
  void initialize_infiltration() {
    infiltration = false;
    if (!precip) return;
    if (qinf > 0.0f) {
      inftype = "con";
      infiltration = true;
    } else if (qinffile.substr(0, 4) != "none") {
      inftype = "c2d";
      infiltration = true;
    } else if (infiltrationfile != "none") {
      throw std::runtime_error("oracle: netCDF infiltration files are not restated");
    } else if (scsfile != "none") {
      inftype = "cna";
      infiltration = true;
      store_cumulative_precipitation = true;
    } else if (sefffile != "none") {
      inftype = "cnb";
      infiltration = true;
      store_cumulative_precipitation = true;
    } else if (psifile != "none") {
      inftype = "gai";
      infiltration = true;
    } else if (f0file != "none") {
      inftype = "hor";
      infiltration = true;
    }
    cumprcp.alloc(np);
    cuminf.alloc(np);
    if (!infiltration) return;
    qinffield.alloc(np);
    qinfmap.alloc(np);
    auto rd = [&](const std::string& f) { return read_stream<float>(path(f), (size_t)np); };
    if (inftype == "cna") {  // :249-279, S from inches to m
      auto r = rd(scsfile);
      for (long nm = 1; nm <= np; nm++) qinffield(nm) = r[nm - 1] * 0.0254f;
      return;
    }
    if (inftype == "cnb") {  // :280-360
      auto smax = rd(smaxfile), se = rd(sefffile), ks = rd(ksfile);
      scs_Se.alloc(np); ksfield.alloc(np); inf_kr.alloc(np);
      scs_P1.alloc(np); scs_F1.alloc(np); rain_T1.alloc(np); scs_S1.alloc(np); scs_rain.alloc(np);
      for (long nm = 1; nm <= np; nm++) {
        qinffield(nm) = smax[nm - 1];
        scs_Se(nm) = se[nm - 1];
        ksfield(nm) = ks[nm - 1];
        inf_kr(nm) = std::sqrt(ksfield(nm) / 25.4f) / 75.0f;  // Equation 4-36 (ks in mm/h)
      }
      return;
    }
    if (inftype == "gai") {  // :361-505
      auto psi = rd(psifile), sig = rd(sigmafile), ks = rd(ksfile);
      GA_head.alloc(np); GA_sigma_max.alloc(np); ksfield.alloc(np); inf_kr.alloc(np); rain_T1.alloc(np);
      GA_sigma.alloc(np); GA_F.alloc(np); GA_Lu.alloc(np);
      for (long nm = 1; nm <= np; nm++) {
        GA_head(nm) = psi[nm - 1];
        GA_sigma_max(nm) = sig[nm - 1];
        ksfield(nm) = ks[nm - 1];
        inf_kr(nm) = std::sqrt(ksfield(nm) / 25.4f) / 75.0f;
        GA_sigma(nm) = GA_sigma_max(nm);
        GA_Lu(nm) = 4.0f * std::sqrt(25.4f) * std::sqrt(ksfield(nm));  // Equation 4-33
        GA_head(nm) = GA_head(nm) / 1000.0f;
        GA_Lu(nm) = GA_Lu(nm) / 1000.0f;
        ksfield(nm) = ksfield(nm) / 1000.0f / 3600.0f;
      }
      return;
    }
    if (inftype == "hor") {  // :506-590
      auto fc = rd(fcfile), f0 = rd(f0file), kd = rd(kdfile);
      horton_fc.alloc(np); horton_f0.alloc(np); horton_kd.alloc(np); rain_T1.alloc(np);
      for (long nm = 1; nm <= np; nm++) {
        horton_fc(nm) = fc[nm - 1];
        horton_f0(nm) = f0[nm - 1];
        horton_kd(nm) = kd[nm - 1];
        qinffield(nm) = horton_f0(nm) / 3600.0f / 1000.0f;
      }
      return;
    }
    if (inftype == "con") {
      for (long nm = 1; nm <= np; nm++) {
        float zz = subgrid ? sg_z_zmin(nm) : zb(nm);
        qinffield(nm) = zz > qinf_zmin ? qinf : 0.0f;
      }
    } else {
      auto r = read_stream<float>(path(qinffile), (size_t)np);
      for (long nm = 1; nm <= np; nm++) qinffield(nm) = r[nm - 1] / 3600.0f / 1000.0f;
    }
  }

  // initialize_hydro + set_initial_conditions + compute_initial_subgrid_volumes:
  // sfincs_domain.f90:2183-2410, sfincs_initial_conditions.F90:14-180, sfincs_subgrid.F90:907-962
  void initialize_hydro() {
    zs.alloc(np);
    q.alloc(npuv + ncuv + 1);
    q0.alloc(npuv + ncuv + 1);
    uv.alloc(npuv + ncuv + 1);
    uv0.alloc(npuv + ncuv + 1);
    kfuv.alloc(npuv);
    if (wiggle_suppression) {
      zs0.alloc(np);
      zsderv.alloc(np);
    }
    if (store_maximum_waterlevel) zsmax.alloc(np);
    if (store_maximum_velocity) vmax.alloc(np);
    if (store_maximum_flux) qmax.alloc(np);
    if (store_twet) twet.alloc(np);
    if (store_t_zsmax) t_zsmax.alloc(np);
    // set_initial_conditions / read_binary_restart_file: sfincs_initial_conditions.F90:14-268
    std::vector<float> inizs4, iniq;
    if (rstfile.substr(0, 4) == "none" && zsinifile.substr(0, 4) != "none") {
      // read_zsini_file (:270-288): np real*4 levels in cell order, widened to real*8
      if (zsinifile.size() >= 2 && zsinifile.substr(zsinifile.size() - 2) == "nc")
        throw std::runtime_error("oracle: netCDF ini files are not restated");
      inizs4 = read_stream<float>(path(zsinifile), (size_t)np);
    }
    if (rstfile.substr(0, 4) != "none") {
      std::ifstream fin(path(rstfile), std::ios::binary);
      if (!fin) throw std::runtime_error("oracle: cannot open " + rstfile);
      auto rd = [&](void* p, size_t n) {
        fin.read((char*)p, (std::streamsize)n);
        if (!fin) throw std::runtime_error("oracle: restart file too short");
      };
      float rdummy;
      int32_t rsttype = 0;
      rd(&rdummy, 4);
      rd(&rsttype, 4);
      rd(&rdummy, 4);
      if (rsttype >= 1 && rsttype <= 6) {
        inizs4.resize((size_t)np);
        rd(&rdummy, 4);
        rd(inizs4.data(), 4 * (size_t)np);
        rd(&rdummy, 4);
        if (rsttype != 3) {
          iniq.resize((size_t)(npuv + ncuv + 1));
          rd(&rdummy, 4);
          rd(iniq.data(), 4 * iniq.size());
          rd(&rdummy, 4);
          rd(&rdummy, 4);
          for (long ib = 1; ib <= nkcuv2; ib++) rd(&uvmean(ib), 4);
          rd(&rdummy, 4);
        }
        // the infiltration state (:237-258); the arrays exist only with that method
        auto state = [&](F1<float>& a, const char* what) {
          if (!a.allocated()) throw std::runtime_error(std::string("oracle: restart file carries ") + what +
                                                       " but the model does not use that infiltration method");
          rd(&rdummy, 4);
          rd(&a(1), 4 * (size_t)np);
        };
        if (rsttype == 4) state(scs_Se, "scs_Se");
        if (rsttype == 5) {
          state(GA_sigma, "GA_sigma");
          state(GA_F, "GA_F");
        }
        if (rsttype == 6) state(rain_T1, "rain_T1");
      }
    }
    for (long nm = 1; nm <= np; nm++) {
      double inizs = inizs4.empty() ? (double)zini : (double)inizs4[(size_t)nm - 1];
      if (subgrid)
        zs(nm) = (TZ)std::max((double)sg_z_zmin(nm), inizs);
      else
        zs(nm) = (TZ)std::max((double)zb(nm), inizs);
    }
    if (wiggle_suppression)
      for (long nm = 1; nm <= np; nm++) zs0(nm) = (T)zs(nm);
    // combined uv points keep q = uv = 0 until the first momentum step (a
    // restart sets the npuv regular points only, :110-113)
    if (store_maximum_waterlevel) zsmax.fill((T)-999.0f);
    tmaxout = dtmaxout > 1.0e-6f ? (double)t0out + (double)dtmaxout : 1.0e9;  // sfincs_output.f90:30-38
    if (store_maximum_velocity) vmax.fill((T)-999.0f);
    if (store_twet) twet.fill((T)0.0f);
    if (store_t_zsmax) t_zsmax.fill(-999.0f);
    uv.fill((T)0);
    if (!iniq.empty()) {  // fluxes from the restart file and the velocities they imply
      for (long ip = 1; ip <= npuv; ip++) {
        q(ip) = (T)iniq[(size_t)ip - 1];
        long nm = uv_index_z_nm(ip), nmu = uv_index_z_nmu(ip);
        float zsuv = (float)std::max(zs(nm), zs(nmu));
        bool iok = subgrid ? zsuv > sg_uv_zmin(ip) + huthresh : zsuv > zbuvmx(ip);
        if (!iok) continue;
        float huv;
        if (subgrid) {
          if (zsuv > sg_uv_zmax(ip) - 1.0e-4f) {
            huv = sg_uv_havg_zmax(ip) + zsuv;
          } else {
            float dzuv = (sg_uv_zmax(ip) - sg_uv_zmin(ip)) / (float)(subgrid_nlevels - 1);
            long iuv = (long)((zsuv - sg_uv_zmin(ip)) / dzuv) + 1;
            float facint = (zsuv - (sg_uv_zmin(ip) + (float)(iuv - 1) * dzuv)) / dzuv;
            huv = sg_uv_havg(iuv, ip) + (sg_uv_havg(iuv + 1, ip) - sg_uv_havg(iuv, ip)) * facint;
          }
          huv = std::max(huv, huthresh);
        } else {
          huv = std::max(zsuv - zbuv(ip), huthresh);
        }
        uv(ip) = (T)std::max(std::min((float)q(ip) / huv, 4.0f), -4.0f);
      }
    }
    if (wind) {
      tauwu.alloc(np);
      tauwv.alloc(np);
      tauwu0.alloc(np);
      tauwu1.alloc(np);
      tauwv0.alloc(np);
      tauwv1.alloc(np);
    }
    if (precip) {
      prcp.alloc(np);
      netprcp.alloc(np);
      prcp0.alloc(np);
      prcp1.alloc(np);
    }
    if (patmos) {  // sfincs_domain.f90:2354-2366
      patm.alloc(np);
      patm0.alloc(np);
      patm1.alloc(np);
      if (pavbnd > 0.0f) patmb.alloc(std::max(ngbnd, 1L), 101200.0f);
    }
    twindupd = t0;  // sfincs_lib.f90:290
    if (use_qext) qext.alloc(np);
    if (subgrid) {
      z_volume.alloc(np);
      long L = subgrid_nlevels;
      for (long nm = 1; nm <= np; nm++) {
        if (zs(nm) >= sg_z_zmax(nm)) {
          z_volume(nm) = (TV)((double)sg_z_volmax(nm) + (double)area_of(nm) *
                                                         ((double)zs(nm) - (double)std::max(sg_z_zmax(nm), -20.0f)));
        } else {
          long ivol = 1;
          for (long il = 2; il <= L; il++) {
            if (sg_z_dep(il, nm) > zs(nm)) {
              ivol = il - 1;
              break;
            }
          }
          float dzvol = sg_z_volmax(nm) / (float)(L - 1);
          float facint = (float)(((double)zs(nm) - (double)sg_z_dep(ivol, nm)) /
                                 (double)std::max(sg_z_dep(ivol + 1, nm) - sg_z_dep(ivol, nm), 0.001f));
          z_volume(nm) = (TV)((float)(ivol - 1) * dzvol + facint * dzvol);
        }
      }
    }
  }

  // set_advection_mask: sfincs_domain.f90:2114-2180
  void set_advection_mask() {
    for (long ic = 1; ic <= ncuv; ic++) {
      int a = kcuv(cuv_index_uv1(ic)), b = kcuv(cuv_index_uv2(ic));
      int8_t& k = kcuv(cuv_index_uv(ic));
      if (a == 0 || b == 0)
        k = 0;
      else if (a == 2 || b == 2)
        k = 2;
      else if (a == 4 || b == 4)
        k = 4;
      else
        k = 1;
    }
    if (advection) {
      mask_adv.alloc(npuv, 1);
      if (advection_mask && (use_quadtree || nmax > 1)) {
        for (long ip = 1; ip <= npuv; ip++) {
          if (kcuv(uv_index_u_nmu(ip)) != 1 || kcuv(uv_index_u_nmd(ip)) != 1 || kcuv(uv_index_v_nm(ip)) != 1 ||
              kcuv(uv_index_v_nmu(ip)) != 1 || kcuv(uv_index_v_ndm(ip)) != 1 || kcuv(uv_index_v_ndmu(ip)) != 1 ||
              kcuv(uv_index_u_ndm(ip)) != 1 || kcuv(uv_index_u_num(ip)) != 1)
            mask_adv(ip) = 0;
        }
      }
    }
  }

  // read_boundary_data (bnd/bzs branch) + find_boundary_indices: sfincs_boundaries.f90:8-213, 455-679
  void read_boundary_data() {
    nbnd = 0;
    ntbnd = 0;
    itbndlast = 1;
    if (bndfile.substr(0, 4) != "none") {
      auto xy = read_ascii_table(path(bndfile));
      nbnd = (long)xy.size();
      x_bnd.alloc(nbnd);
      y_bnd.alloc(nbnd);
      for (long n = 1; n <= nbnd; n++) {
        x_bnd(n) = (float)xy[n - 1][0];
        y_bnd(n) = (float)xy[n - 1][1];
      }
      if (bzsfile.substr(0, 4) != "none") {
        auto tb = read_ascii_table(path(bzsfile));
        ntbnd = (long)tb.size();
        t_bnd.alloc(ntbnd);
        zs_bnd.alloc(nbnd, ntbnd);
        zst_bnd.alloc(nbnd);
        for (long it = 1; it <= ntbnd; it++) {
          t_bnd(it) = (float)tb[it - 1][0];
          for (long ib = 1; ib <= nbnd; ib++) zs_bnd(ib, it) = (float)tb[it - 1][ib];
        }
      } else {
        ntbnd = 2;
        t_bnd.alloc(2);
        zs_bnd.alloc(nbnd, 2);
        zst_bnd.alloc(nbnd);
        t_bnd(1) = t0;
        t_bnd(2) = t1;
      }
      if (t_bnd(1) > (t0 + 1.0f) || t_bnd(ntbnd) < (t1 - 1.0f)) {
        if (t_bnd(1) > (t0 + 1.0f))
          t_bnd(1) = t0 - 1.0f;
        else
          t_bnd(ntbnd) = t1 + 1.0f;
      }
    } else if (water_level_boundaries_in_mask) {
      nbnd = 1;
      x_bnd.alloc(1);
      y_bnd.alloc(1);
      ntbnd = 2;
      t_bnd.alloc(2);
      zs_bnd.alloc(1, 2);
      zst_bnd.alloc(1);
      t_bnd(1) = t0;
      t_bnd(2) = t1;
    }
    nr_tidal_components = 0;
    if (bcafile.substr(0, 4) != "none" && nbnd > 0 && use_bcafile) read_bca();
    // downstream river points: x, y, internal x, y, slope, distance per line (:217-270)
    nbdr = 0;
    if (downstream_river_boundaries_in_mask) {
      if (bdrfile.substr(0, 4) == "none")
        throw std::runtime_error("oracle: downstream river points in the mask without a bdrfile");
      auto rows = read_ascii_table(path(bdrfile));
      nbdr = (long)rows.size();
      x_bdr.alloc(nbdr);
      y_bdr.alloc(nbdr);
      index_zsi_bdr.alloc(nbdr);
      dzs_bdr.alloc(nbdr);
      for (long i = 1; i <= nbdr; i++) {
        const auto& r = rows[i - 1];
        x_bdr(i) = (float)r.at(0);
        y_bdr(i) = (float)r.at(1);
        float xin = (float)r.at(2), yin = (float)r.at(3), slope = (float)r.at(4), dist = (float)r.at(5);
        long nmq = find_quadtree_cell(xin, yin);
        index_zsi_bdr(i) = nmq > 0 ? index_sfincs_in_quadtree(nmq) : 0;
        if (index_zsi_bdr(i) == 0) throw std::runtime_error("oracle: river point outside the active mesh");
        if (dist < 0.0f)
          dzs_bdr(i) = -slope * std::sqrt((xin - x_bdr(i)) * (xin - x_bdr(i)) + (yin - y_bdr(i)) * (yin - y_bdr(i)));
        else
          dzs_bdr(i) = -slope * dist;
      }
    }
  }

  void find_boundary_indices() {
    if (ngbnd == 0) return;
    if (nbnd == 0 && nbdr == 0) return;
    ind1_bnd_gbp.alloc(ngbnd);
    ind2_bnd_gbp.alloc(ngbnd);
    fac_bnd_gbp.alloc(ngbnd);
    if (downstream_river_boundaries_in_mask) index_bdr_gbp.alloc(ngbnd);
    if (neumann_boundaries_in_mask) nmi_gbp.alloc(ngbnd);
    for (long ib = 1; ib <= ngbnd; ib++) {
      long nm = nmindbnd(ib);
      float x = z_xz(nm), y = z_yz(nm);
      if (kcs(nm) == 2) {
        if (nbnd > 1) {
          float dst1 = 1.0e10f, dst2 = 1.0e10f;
          long ib1 = 0, ib2 = 0;
          for (long ibnd = 1; ibnd <= nbnd; ibnd++) {
            float ddx = x_bnd(ibnd) - x, ddy = y_bnd(ibnd) - y;
            float dst = std::sqrt(ddx * ddx + ddy * ddy);
            if (dst < dst1) {
              dst2 = dst1;
              ib2 = ib1;
              dst1 = dst;
              ib1 = ibnd;
            } else if (dst < dst2) {
              dst2 = dst;
              ib2 = ibnd;
            }
          }
          ind1_bnd_gbp(ib) = (int32_t)ib1;
          ind2_bnd_gbp(ib) = (int32_t)ib2;
          fac_bnd_gbp(ib) = dst2 / std::max(dst1 + dst2, 1.0e-9f);
        } else {
          ind1_bnd_gbp(ib) = 1;
          ind2_bnd_gbp(ib) = 1;
          fac_bnd_gbp(ib) = 1.0f;
        }
      } else if (kcs(nm) == 5) {  // nearest point of the bdr file (:596-613)
        float dst1 = 1.0e10f;
        long ib1 = 0;
        for (long ibdr = 1; ibdr <= nbdr; ibdr++) {
          float ddx = x_bdr(ibdr) - x, ddy = y_bdr(ibdr) - y;
          float dst = std::sqrt(ddx * ddx + ddy * ddy);
          if (dst < dst1) {
            dst1 = dst;
            ib1 = ibdr;
          }
        }
        index_bdr_gbp(ib) = (int32_t)ib1;
      } else if (kcs(nm) == 6) {
        // regular grid: find_sfincs_cell(n, m+-1 / n+-1, iref) through the quadtree search arrays
        long n = z_index_z_n(nm), m = z_index_z_m(nm);
        auto find = [&](long nn, long mm) -> long {
          long nmq = find_qt_by_index(nn, mm, z_flags_iref(nm));
          return nmq > 0 ? index_sfincs_in_quadtree(nmq) : 0;
        };
        long cand[4][2] = {{n, m + 1}, {n + 1, m}, {n, m - 1}, {n - 1, m}};
        for (auto& c : cand) {
          long nmi = find(c[0], c[1]);
          if (nmi > 0 && kcs(nmi) == 1) nmi_gbp(ib) = (int32_t)nmi;
        }
        if (nmi_gbp(ib) == 0) kcs(nm) = 0;
      }
    }
  }

  // read_thin_dams: sfincs_structures.f90:385-495.  Polylines of a .thd file
  // (name line, "nrows ncols", nrows lines of x y); every uv point crossed by a
  // polyline segment gets kcuv = 0.
  void read_thin_dams() {
    if (thdfile.substr(0, 4) == "none") return;
    std::ifstream fin(path(thdfile));
    if (!fin) throw std::runtime_error("oracle: cannot open " + thdfile);
    std::vector<std::string> rec;  // list-directed input skips blank records
    for (std::string l; std::getline(fin, l);) {
      for (char& ch : l)
        if (ch == ',' || ch == '\t' || ch == '\r') ch = ' ';
      if (l.find_first_not_of(' ') != std::string::npos) rec.push_back(l);
    }
    size_t ir = 0;
    while (ir + 1 < rec.size()) {
      ir++;  // cdummy
      std::istringstream hs(rec[ir++]);
      int nrows = 0, ncols = 0;
      hs >> nrows >> ncols;
      std::vector<float> xthd(nrows), ythd(nrows);
      for (int i = 0; i < nrows; i++) {
        if (ir >= rec.size()) throw std::runtime_error("oracle: truncated thin dam polyline");
        std::istringstream ps(rec[ir++]);
        ps >> xthd[i] >> ythd[i];
      }
      for (const auto& e : uv_points_crossed_by_polyline(xthd, ythd)) kcuv(e.first) = 0;
    }
  }

  // direction / cross: third_party_open/utils/geometry.f90:121-190 (real*4)
  static int direction(float ax, float ay, float bx, float by, float cx, float cy) {
    float val = (by - ay) * (cx - bx) - (bx - ax) * (cy - by);
    if (val < -1.0e-6f) return -1;
    if (val > 1.0e-6f) return 1;
    return 0;
  }
  static bool cross(float x11, float y11, float x12, float y12, float x21, float y21, float x22, float y22) {
    int dir1 = direction(x11, y11, x12, y12, x21, y21);
    int dir2 = direction(x11, y11, x12, y12, x22, y22);
    int dir3 = direction(x21, y21, x22, y22, x11, y11);
    int dir4 = direction(x21, y21, x22, y22, x12, y12);
    return dir1 != dir2 && dir3 != dir4;
  }

  // find_uv_points_intersected_by_polyline: sfincs_quadtree.F90:853-1010
  // (the crossed uv points, ascending, each with the last segment that
  // crossed it, 1-based: uv_indices and vertices).
  std::vector<std::pair<long, int>> uv_points_crossed_by_polyline(const std::vector<float>& xpol,
                                                                   const std::vector<float>& ypol) {
    std::vector<int> ind((size_t)npuv + 1, 0);
    const long npol = (long)xpol.size();
    for (long ipol = 1; ipol <= npol - 1; ipol++) {
      float xpa = xpol[ipol - 1], ypa = ypol[ipol - 1], xpb = xpol[ipol], ypb = ypol[ipol];
      float xtmpa = qt_cosrot * (xpa - x0) + qt_sinrot * (ypa - y0);
      float ytmpa = -qt_sinrot * (xpa - x0) + qt_cosrot * (ypa - y0);
      float xtmpb = qt_cosrot * (xpb - x0) + qt_sinrot * (ypb - y0);
      float ytmpb = -qt_sinrot * (xpb - x0) + qt_cosrot * (ypb - y0);
      for (int iref = qt_nlev; iref >= 1; iref--) {
        long na = (long)(ytmpa / qt_dyr(iref)) + 1, ma = (long)(xtmpa / qt_dxr(iref)) + 1;
        long nb = (long)(ytmpb / qt_dyr(iref)) + 1, mb = (long)(xtmpb / qt_dxr(iref)) + 1;
        long n0 = std::min(na, nb) - 1, n1 = std::max(na, nb) + 1, m0 = std::min(ma, mb) - 1, m1 = std::max(ma, mb) + 1;
        for (long m = m0; m <= m1; m++) {
          for (long n = n0; n <= n1; n++) {
            long nm = find_qt_by_index_unchecked(n, m, iref);
            if (nm == 0) continue;
            nm = index_sfincs_in_quadtree(nm);
            if (nm == 0) continue;
            for (long ip : {(long)z_index_uv_mu1(nm), (long)z_index_uv_mu2(nm), (long)z_index_uv_nu1(nm),
                            (long)z_index_uv_nu2(nm)}) {
              if (ip <= 0) continue;
              long nmu = uv_index_z_nmu(ip);
              if (cross(xpa, ypa, xpb, ypb, z_xz(nm), z_yz(nm), z_xz(nmu), z_yz(nmu))) ind[(size_t)ip] = (int)ipol;
            }
          }
        }
      }
    }
    std::vector<std::pair<long, int>> out;
    for (long ip = 1; ip <= npuv; ip++)
      if (ind[(size_t)ip] > 0) out.push_back({ip, ind[(size_t)ip]});
    return out;
  }

  // read_crs_file: sfincs_crosssections.f90:8-127.  Polylines of the crs
  // file; per polyline the uv points it crosses and the sign of each crossing
  // from the angle between the uv point's direction and the segment.
  std::string crsfile = "none";
  std::vector<std::string> namecrs;
  std::vector<std::vector<long>> crs_uv_index;
  std::vector<std::vector<int>> crs_idir;
  void read_crs_file() {
    if (crsfile.substr(0, 4) == "none") return;
    std::ifstream fin(path(crsfile));
    if (!fin) throw std::runtime_error("oracle: cannot open " + crsfile);
    std::vector<std::string> rec;
    for (std::string l; std::getline(fin, l);) {
      for (char& ch : l)
        if (ch == ',' || ch == '\t' || ch == '\r') ch = ' ';
      if (l.find_first_not_of(' ') != std::string::npos) rec.push_back(l);
    }
    size_t ir = 0;
    while (ir + 1 < rec.size()) {
      std::string cdummy;  // list-directed: the first item, a quoted string whole
      {
        const std::string& l = rec[ir++];
        const size_t a = l.find_first_not_of(' ');
        if (l[a] == '\'' || l[a] == '"') {
          const size_t b = l.find(l[a], a + 1);
          cdummy = l.substr(a + 1, (b == std::string::npos ? l.size() : b) - a - 1);
        } else {
          std::istringstream(l) >> cdummy;
        }
      }
      std::istringstream hs(rec[ir++]);
      int nrows = 0, ncols = 0;
      hs >> nrows >> ncols;
      std::vector<float> xcrs(nrows), ycrs(nrows);
      for (int i = 0; i < nrows; i++) {
        if (ir >= rec.size()) throw std::runtime_error("oracle: truncated cross-section polyline");
        std::istringstream ps(rec[ir++]);
        ps >> xcrs[i] >> ycrs[i];
      }
      namecrs.push_back(cdummy);
      std::vector<long> idx;
      std::vector<int> idir;
      for (const auto& e : uv_points_crossed_by_polyline(xcrs, ycrs)) {
        const long indx = e.first, irow = e.second;
        const long nm = uv_index_z_nm(indx), nmu = uv_index_z_nmu(indx);
        const float phiuv = std::atan2(z_yz(nmu) - z_yz(nm), z_xz(nmu) - z_xz(nm));
        const float phic = std::atan2(ycrs[irow] - ycrs[irow - 1], xcrs[irow] - xcrs[irow - 1]);
        float dphi = phiuv - phic;
        if (dphi < 0.0f) dphi = dphi + 2 * pi;
        if (dphi > 2 * pi) dphi = dphi - 2 * pi;
        idx.push_back(indx);
        idir.push_back(dphi <= pi ? 1 : -1);
      }
      crs_uv_index.push_back(idx);
      crs_idir.push_back(idir);
    }
  }

  // read_rug_file: sfincs_runup_gauges.f90:3-115 (two points per gauge, a
  // point every 0.2 finest cell widths, its cell by find_quadtree_cell)
  std::string rugfile = "none";
  float runup_gauge_depth = 0.05f;
  std::vector<std::vector<long>> runup_gauge_nm;
  void read_rug_file() {
    if (rugfile.substr(0, 4) == "none") return;
    std::ifstream fin(path(rugfile));
    if (!fin) throw std::runtime_error("oracle: cannot open " + rugfile);
    std::vector<std::string> rec;
    for (std::string l; std::getline(fin, l);) {
      for (char& ch : l)
        if (ch == ',' || ch == '\t' || ch == '\r') ch = ' ';
      if (l.find_first_not_of(' ') != std::string::npos) rec.push_back(l);
    }
    const float dxstep = 0.2f * dxyr(nref);
    size_t ir = 0;
    while (ir + 3 < rec.size() + 1 && ir + 1 < rec.size()) {
      ir++;  // name
      std::istringstream hs(rec[ir++]);
      int nrows = 0, ncols = 0;
      hs >> nrows >> ncols;
      if (nrows != 2 || ir + 2 > rec.size()) throw std::runtime_error("oracle: run-up gauge needs two points");
      float xru0, yru0, xru1, yru1;
      std::istringstream(rec[ir++]) >> xru0 >> yru0;
      std::istringstream(rec[ir++]) >> xru1 >> yru1;
      const float rdx = xru1 - xru0, rdy = yru1 - yru0;
      const float rlen = std::sqrt(rdx * rdx + rdy * rdy);
      const long nrp = (long)(rlen / dxstep) + 1;
      std::vector<long> nms;
      for (long ip = 1; ip <= nrp; ip++) {
        const float x = xru0 + (float)(ip - 1) * dxstep * rdx / rlen;
        const float y = yru0 + (float)(ip - 1) * dxstep * rdy / rlen;
        const long nmq = find_quadtree_cell(x, y);
        const long nm = nmq > 0 ? index_sfincs_in_quadtree(nmq) : 0;
        if (nm <= 0) throw std::runtime_error("oracle: run-up gauge point outside the mesh");
        nms.push_back(nm);
      }
      runup_gauge_nm.push_back(nms);
    }
  }

  // get_runup_levels: sfincs_runup_gauges.f90:117-150
  float runup_level(size_t irug) {
    float zru = -999.0f;
    for (long nm : runup_gauge_nm[irug]) {
      const float zbt = subgrid ? (float)sg_z_zmin(nm) : (float)zb(nm);
      if ((double)zs(nm) > (double)(zbt + runup_gauge_depth)) zru = (float)zs(nm);
    }
    return zru;
  }

  // get_discharges_through_crosssections: sfincs_crosssections.f90:130-176
  float crs_discharge(size_t icrs) {
    float qq = 0.0f;
    for (size_t ip = 0; ip < crs_uv_index[icrs].size(); ip++) {
      const long indx = crs_uv_index[icrs][ip];
      const int iref = uv_flags_iref(indx), iuv = uv_flags_dir(indx);
      const float dxycrs = iuv == 0 ? dyrm(iref) : dxrm(iref);
      qq = qq + (float)q(indx) * (float)crs_idir[icrs][ip] * dxycrs;
    }
    return qq;
  }

  // read_structures: sfincs_structures.f90:8-35 (thin dams, then weirs)
  void read_structures() {
    read_thin_dams();
    nrstructures = 0;
    if (weirfile.substr(0, 4) != "none") read_structure_file(weirfile, 1, 2);
  }

  // distance_between_points_projected_on_line_segment:
  // third_party_open/utils/geometry.f90:215-297 (real*4)
  static float projected_distance(float x0a, float y0a, float x0b, float y0b, float x1, float y1, float x2, float y2,
                                  float mxdst) {
    float b1, b2, c1, c2, aa, a1, a2, p1, p2;
    b1 = std::fabs((x2 - x1) * (y1 - y0a) - (x1 - x0a) * (y2 - y1)) / (std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)));
    c1 = std::sqrt((x0a - x1) * (x0a - x1) + (y0a - y1) * (y0a - y1));
    c2 = std::sqrt((x0a - x2) * (x0a - x2) + (y0a - y2) * (y0a - y2));
    aa = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    a1 = std::sqrt(std::max(c1 * c1 - b1 * b1, 0.0f));
    a2 = std::sqrt(std::max(c2 * c2 - b1 * b1, 0.0f));
    if (a1 > aa || a2 > aa)
      p1 = a1 < a2 ? 0.0f : 1.0f;
    else
      p1 = a1 / aa;
    b2 = std::fabs((x2 - x1) * (y1 - y0b) - (x1 - x0b) * (y2 - y1)) / (std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)));
    c1 = std::sqrt((x0b - x1) * (x0b - x1) + (y0b - y1) * (y0b - y1));
    c2 = std::sqrt((x0b - x2) * (x0b - x2) + (y0b - y2) * (y0b - y2));
    aa = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    a1 = std::sqrt(std::max(c1 * c1 - b2 * b2, 0.0f));
    a2 = std::sqrt(std::max(c2 * c2 - b2 * b2, 0.0f));
    if (a1 > aa || a2 > aa)
      p2 = a1 < a2 ? 0.0f : 1.0f;
    else
      p2 = a1 / aa;
    return (b1 < mxdst && b2 < mxdst) ? aa * std::fabs(p2 - p1) : 0.0f;
  }

  // read_structure_file: sfincs_structures.f90:38-381 (projected grids)
  void read_structure_file(const std::string& filename, int itype, int npars) {
    std::ifstream fin(path(filename));
    if (!fin) throw std::runtime_error("oracle: cannot open " + filename);
    std::vector<std::string> rec;
    for (std::string l; std::getline(fin, l);) {
      for (char& ch : l)
        if (ch == ',' || ch == '\t' || ch == '\r') ch = ' ';
      if (l.find_first_not_of(' ') != std::string::npos) rec.push_back(l);
    }
    F1<int8_t> istruc;
    istruc.alloc(npuv);
    F2<float> strucpars;
    strucpars.alloc(npars, npuv);
    for (long ip = 1; ip <= npuv; ip++) strucpars(1, ip) = -9999.0f;
    F1<float> lngth;
    lngth.alloc(npuv);
    size_t ir = 0;
    while (ir + 1 < rec.size()) {
      ir++;  // cdummy
      std::istringstream hs(rec[ir++]);
      int nrows = 0, ncols = 0;
      hs >> nrows >> ncols;
      std::vector<float> xthd(nrows), ythd(nrows);
      std::vector<std::vector<float>> pars(npars + 1, std::vector<float>(nrows + 1));
      for (int irow = 1; irow <= nrows; irow++) {
        if (ir >= rec.size()) throw std::runtime_error("oracle: truncated structure polyline");
        std::istringstream ps(rec[ir++]);
        ps >> xthd[irow - 1] >> ythd[irow - 1];
        for (int ipar = 1; ipar <= npars; ipar++) ps >> pars[ipar][irow];
      }
      for (const auto& e : uv_points_crossed_by_polyline(xthd, ythd)) {
        long indx = e.first;
        int irow = e.second;
        istruc(indx) = 1;
        long nm = uv_index_z_nm(indx), nmu = uv_index_z_nmu(indx);
        int iref = uv_flags_iref(indx), idir = uv_flags_dir(indx);
        int irefnm = z_flags_iref(nm), irefnmu = z_flags_iref(nmu);
        float dxs = idir == 0 ? dyrm(iref) : dxrm(iref);
        float xuv, yuv, xuv1, yuv1, xuv2, yuv2;
        if (irefnm >= irefnmu) {
          if (idir == 0) {
            xuv = z_xz(nm) + 0.5f * dxs * std::cos(rotation);
            yuv = z_yz(nm) + 0.5f * dxs * std::sin(rotation);
          } else {
            xuv = z_xz(nm) + 0.5f * dxs * std::cos(rotation + 0.5f * pi);
            yuv = z_yz(nm) + 0.5f * dxs * std::sin(rotation + 0.5f * pi);
          }
        } else {
          if (idir == 0) {
            xuv = z_xz(nmu) + 0.5f * dxs * std::cos(rotation - pi);
            yuv = z_yz(nmu) + 0.5f * dxs * std::sin(rotation - pi);
          } else {
            xuv = z_xz(nmu) + 0.5f * dxs * std::cos(rotation - 0.5f * pi);
            yuv = z_yz(nmu) + 0.5f * dxs * std::sin(rotation - 0.5f * pi);
          }
        }
        if (idir == 0) {
          xuv1 = xuv + 0.5f * dxs * std::cos(rotation - 0.5f * pi);
          yuv1 = yuv + 0.5f * dxs * std::sin(rotation - 0.5f * pi);
          xuv2 = xuv + 0.5f * dxs * std::cos(rotation + 0.5f * pi);
          yuv2 = yuv + 0.5f * dxs * std::sin(rotation + 0.5f * pi);
        } else {
          xuv1 = xuv + 0.5f * dxs * std::cos(rotation - pi);
          yuv1 = yuv + 0.5f * dxs * std::sin(rotation - pi);
          xuv2 = xuv + 0.5f * dxs * std::cos(rotation);
          yuv2 = yuv + 0.5f * dxs * std::sin(rotation);
        }
        float d = projected_distance(xuv1, yuv1, xuv2, yuv2, xthd[irow - 1], ythd[irow - 1], xthd[irow], ythd[irow],
                                     999999.0f);
        lngth(indx) = lngth(indx) + d;
        float dst1 = std::sqrt((xuv - xthd[irow - 1]) * (xuv - xthd[irow - 1]) + (yuv - ythd[irow - 1]) * (yuv - ythd[irow - 1]));
        float dst2 = std::sqrt((xuv - xthd[irow]) * (xuv - xthd[irow]) + (yuv - ythd[irow]) * (yuv - ythd[irow]));
        float wfac = dst1 / (dst1 + dst2);
        float height = pars[1][irow] * (1.0f - wfac) + pars[1][irow + 1] * wfac;
        strucpars(1, indx) = std::max(strucpars(1, indx), height);
        for (int ipar = 2; ipar <= npars; ipar++)
          strucpars(ipar, indx) = pars[ipar][irow] * (1.0f - wfac) + pars[ipar][irow + 1] * wfac;
      }
    }
    long nstruc = 0;
    for (long ip = 1; ip <= npuv; ip++) {
      bool okay = false;
      if (istruc(ip) == 1) {
        float height = strucpars(1, ip);
        if (subgrid) {
          if (height > sg_uv_zmin(ip)) okay = true;
        } else {
          if (height > zbuvmx(ip)) okay = true;
        }
      }
      if (okay)
        nstruc++;
      else
        istruc(ip) = 0;
    }
    structure_uv_index.alloc(nstruc);
    structure_type.alloc(nstruc);
    structure_length.alloc(nstruc);
    structure_parameters.alloc(npars, nstruc);
    nstruc = 0;
    for (long ip = 1; ip <= npuv; ip++) {
      if (istruc(ip) != 1) continue;
      nstruc++;
      structure_type(nstruc) = (int8_t)itype;
      structure_uv_index(nstruc) = (int32_t)ip;
      int iref = uv_flags_iref(ip), idir = uv_flags_dir(ip);
      float dxs = idir == 0 ? dyrm(iref) : dxrm(iref);
      structure_length(nstruc) = lngth(ip) / dxs;
      for (int ipar = 1; ipar <= npars; ipar++) structure_parameters(ipar, nstruc) = strucpars(ipar, ip);
      kcuv(ip) = 3;
    }
    nrstructures = nstruc;
  }

  // compute_fluxes_over_structures: sfincs_structures.f90:592-697
  void compute_fluxes_over_structures() {
    for (long istruc = 1; istruc <= nrstructures; istruc++) {
      long ip = structure_uv_index(istruc);
      q(ip) = (T)0;
      uv(ip) = (T)0;
      long nm = uv_index_z_nm(ip), nmu = uv_index_z_nmu(ip);
      T zsnm = (T)zs(nm), zsnmu = (T)zs(nmu);
      T height = (T)structure_parameters(1, istruc);
      if (zsnm < height && zsnmu < height) continue;
      T qstruc = (T)0;
      int idir = 1;
      if (structure_type(istruc) == 1) {
        T cweir = (T)1.7049f, m = (T)0, Cd = (T)structure_parameters(2, istruc), h1, h2;
        if (zsnm > zsnmu) {
          idir = 1;
          h1 = zsnm - height;
          h2 = zsnmu - height;
        } else {
          idir = -1;
          h1 = zsnmu - height;
          h2 = zsnm - height;
        }
        if (h2 > (T)(2.0f / 3.0f) * h1)
          qstruc = Cd * h2 * std::sqrt((T)2.0f * (T)9.81f * (h1 - h2) / ((T)1 - m));
        else  // h1**1.5; the core's precision evaluates it as h1 * sqrt(h1), correctly rounded on CPU and GPU alike
          qstruc = Cd * cweir * (std::is_same<TZ, float>::value ? h1 * std::sqrt(h1) : std::pow(h1, (T)1.5f));
      }
      qstruc = qstruc * (T)structure_length(istruc);
      q(ip) = qstruc * (T)idir;
    }
  }

  // find_quadtree_cell_by_index as written (sfincs_quadtree.F90:822-850): no
  // check of n against the level's row count, only nm > 0; a miss returns
  // binary_search's 0 shifted by the level's first index minus one (0 on
  // level 1, the only level of a regular grid).
  long find_qt_by_index_unchecked(long n, long m, int iref) {
    long nmx = (long)qt_nmax << (iref - 1);
    long nm = (m - 1) * nmx + n;
    if (nm <= 0) return 0;
    long i1 = qt_first(iref), i2 = qt_last(iref);
    long lo = 0, hi = i2 - i1 + 1, found = 0;  // binary_search(x(i1:i2), n, val): 1-based, middle 0 skipped
    while (lo <= hi && !found) {
      long mid = (lo + hi) / 2;
      if (mid == 0)
        lo = mid + 1;
      else if (nm == qt_nm_indices(i1 + mid - 1))
        found = mid;
      else if (nm < qt_nm_indices(i1 + mid - 1))
        hi = mid - 1;
      else
        lo = mid + 1;
    }
    return found + i1 - 1;
  }

  // find_quadtree_cell_by_index + binary_search: sfincs_quadtree.F90:822-850
  long find_qt_by_index(long n, long m, int iref) {
    long nmx = (long)qt_nmax << (iref - 1);
    long nm = (m - 1) * nmx + n;
    long i1 = qt_first(iref), i2 = qt_last(iref);
    if (nm <= 0 || n < 1 || m < 1) return 0;
    long lo = i1, hi = i2;
    while (lo <= hi) {
      long mid = (lo + hi) / 2;
      long v = qt_nm_indices(mid);
      if (v == nm) return mid;
      if (v < nm)
        lo = mid + 1;
      else
        hi = mid - 1;
    }
    return 0;
  }

  // read_meteo_data (time-series part) + Cd table: sfincs_meteo.f90:247-327
  // read_amuv_dimensions + read_amuv_file: sfincs_spiderweb.f90:135-230, 320-403.
  // Header keys up to the first line that starts with TIME, then per time a
  // TIME line and nrows x ncols values (list-directed), rows from the top.
  void read_am_file(const std::string& file, AmGrid& g, int q) {
    std::ifstream fin(path(file));
    if (!fin) throw std::runtime_error("oracle: cannot open " + file);
    std::vector<std::string> lines;
    for (std::string l; std::getline(fin, l);) {
      if (!l.empty() && l.back() == '\r') l.pop_back();
      lines.push_back(l);
    }
    size_t i = 0;
    std::map<std::string, std::string> kv;
    for (; i < lines.size() && lines[i].compare(0, 4, "TIME") != 0; i++) {
      size_t e = lines[i].find('=');
      if (e == std::string::npos) continue;
      std::string k = lines[i].substr(0, e), v = lines[i].substr(e + 1);
      k.erase(0, k.find_first_not_of(" \t"));
      k.erase(k.find_last_not_of(" \t") + 1);
      for (auto& ch : k) ch = (char)std::tolower(ch);
      kv[k] = v;
    }
    auto num = [&](const char* k) {
      auto it = kv.find(k);
      return it == kv.end() ? 0.0 : std::strtod(it->second.c_str(), nullptr);
    };
    const int ncols = (int)num("n_cols"), nrows = (int)num("n_rows");
    const float x_ll = (float)num("x_llcorner"), y_ll = (float)num("y_llcorner"), ddx = (float)num("dx"),
                ddy = (float)num("dy");
    if (ncols < 1 || nrows < 1) throw std::runtime_error("oracle: meteo file without n_cols / n_rows: " + file);
    std::vector<float> times, vals;
    while (i < lines.size()) {
      if (lines[i].compare(0, 4, "TIME") != 0) {
        i++;
        continue;
      }
      times.push_back(meteo_time_seconds(lines[i], trefstr));
      i++;
      size_t need = (size_t)nrows * ncols, got = 0;
      while (got < need && i < lines.size()) {
        std::istringstream ls(lines[i++]);
        double x;
        while (got < need && ls >> x) {
          vals.push_back((float)x);
          got++;
        }
      }
      if (got < need) throw std::runtime_error("oracle: truncated meteo file " + file);
    }
    if (q == 0) {
      g.nt = (int)times.size();
      g.nrows = nrows;
      g.ncols = ncols;
      g.x_ll = x_ll;
      g.y_ll = y_ll;
      g.dx = ddx;
      g.dy = ddy;
      g.times = times;
    }
    g.v[q] = vals;
  }

  // The window fields (update_amuv_data / update_amp_data / update_ampr_data,
  // sfincs_meteo.f90:802-1243): for each end of the window the two records
  // around it, blended in time on the meteo grid, then bilinear on each cell.
  // kind 0: wind stress from amu/amv, 1: pressure, 2: rain.
  void update_am_window(const AmGrid& g, int kind) {
    for (int itw = 1; itw <= 2; itw++) {
      float meteo_t = itw == 1 ? meteo_t0 : meteo_t1;
      meteo_t = std::max(meteo_t, g.times[0]);
      meteo_t = std::min(meteo_t, g.times[g.nt - 1]);
      int itw0 = 1;
      for (int it = 1; it <= g.nt; it++)
        if (g.times[it - 1] <= meteo_t) itw0 = it;
      const int itw1 = std::min(itw0 + 1, g.nt);
      meteo_t = std::min(meteo_t, g.times[itw1 - 1]);
      float twfac = (meteo_t - g.times[itw0 - 1]) / std::max(g.times[itw1 - 1] - g.times[itw0 - 1], 1.0e-6f);
      if (kind == 2 && ampr_block) twfac = 0.0f;
      auto v01 = [&](int q, int irow, int icol) {
        return g.at(q, itw0, irow, icol) * (1.0f - twfac) + g.at(q, itw1, irow, icol) * twfac;
      };
      const float yul = g.y_ll + (float)(g.nrows - 1) * g.dy + 0.5f * g.dy;
      const float xll = g.x_ll + 0.5f * g.dx;
      for (long nm = 1; nm <= np; nm++) {
        const float x = z_xz(nm), y = z_yz(nm);
        const int iy = (int)((yul - y) / g.dy) + 1;
        const int ind1[4] = {iy, iy, iy + 1, iy + 1};
        const float dj1 = (yul - (float)(iy - 1) * g.dy - y) / g.dy;
        const int ix = (int)((x - xll) / g.dx) + 1;
        const int ind2[4] = {ix, ix + 1, ix + 1, ix};
        const float di1 = (x - (xll + (float)(ix - 1) * g.dx)) / g.dx;
        if (iy <= 1 || iy >= g.nrows || ix <= 0 || ix >= g.ncols) {  // outside the meteo grid
          if (kind == 0) {
            (itw == 1 ? tauwu0 : tauwu1)(nm) = 0.0f;
            (itw == 1 ? tauwv0 : tauwv1)(nm) = 0.0f;
          } else if (kind == 1) {
            (itw == 1 ? patm0 : patm1)(nm) = gapres;
          } else {
            (itw == 1 ? prcp0 : prcp1)(nm) = 0.0f;
          }
          continue;
        }
        const float f[4] = {(1.0f - di1) * (1.0f - dj1), di1 * (1.0f - dj1), di1 * dj1, (1.0f - di1) * dj1};
        if (kind == 0) {
          float wup = 0.0f, wvp = 0.0f;
          for (int ip = 0; ip < 4; ip++) {
            wup = wup + f[ip] * v01(0, ind1[ip], ind2[ip]);
            wvp = wvp + f[ip] * v01(1, ind1[ip], ind2[ip]);
          }
          const float vmag = std::sqrt(wup * wup + wvp * wvp);
          const long icd = std::min(std::max((long)(vmag * 10.0f) + 1, 1L), 1000L);
          const float cd = cdval(icd);
          (itw == 1 ? tauwu0 : tauwu1)(nm) = vmag * (cosrot * wup + sinrot * wvp) * rhoa * cd / rhow;
          (itw == 1 ? tauwv0 : tauwv1)(nm) = vmag * (-sinrot * wup + cosrot * wvp) * rhoa * cd / rhow;
        } else {
          float pr = 0.0f;
          for (int ip = 0; ip < 4; ip++) pr = pr + f[ip] * v01(0, ind1[ip], ind2[ip]);
          if (kind == 1)
            (itw == 1 ? patm0 : patm1)(nm) = pr;
          else
            (itw == 1 ? prcp0 : prcp1)(nm) = pr / (float)(1000 * 3600);
        }
      }
    }
  }

  // read_spw_dimensions + read_spw_file: sfincs_spiderweb.f90:8-134, 231-316.
  // The header keys, the first TIME line within 30 lines (else 16 / 18 header
  // lines), then per record the TIME line, the eye x and y (twelve characters
  // after '='), a skipped line, and nrows rows of ncols values per quantity.
  void read_spw(const std::string& file) {
    std::ifstream fin(path(file));
    if (!fin) throw std::runtime_error("oracle: cannot open " + file);
    std::vector<std::string> lines;
    for (std::string l; std::getline(fin, l);) {
      if (!l.empty() && l.back() == '\r') l.pop_back();
      lines.push_back(l);
    }
    auto key = [&](const char* name) {
      for (const auto& l : lines) {
        size_t e = l.find('=');
        if (e == std::string::npos) continue;
        std::string k = l.substr(0, e);
        k.erase(0, k.find_first_not_of(" \t"));
        k.erase(k.find_last_not_of(" \t") + 1);
        if (k == name) return std::strtod(l.substr(e + 1).c_str(), nullptr);
      }
      return 0.0;
    };
    SpwData& w = spw;
    w.ncols = (int)key("n_cols");
    w.nrows = (int)key("n_rows");
    w.nquant = (int)key("n_quantity");
    w.radius = (float)key("spw_radius");
    long nheader = 0;
    for (long ip = 1; ip <= 30 && ip <= (long)lines.size(); ip++)
      if (lines[ip - 1].find("TIME") == 0) {
        nheader = ip - 1;
        break;
      }
    if (nheader == 0) nheader = w.nquant == 4 ? 18 : 16;
    const long blk = 4 + (long)w.nrows * w.nquant;
    w.nt = (int)(((long)lines.size() - nheader) / blk);
    const size_t rec = (size_t)w.nrows * w.ncols;
    std::vector<float> vmag(rec * w.nt, 0.0f), vdir(rec * w.nt, 0.0f), pdrp(rec * w.nt, 0.0f);
    w.prcp.assign(rec * w.nt, 0.0f);
    long i = nheader;
    auto eye = [&](const std::string& l) { return std::strtof(l.substr(l.find('=') + 1, 12).c_str(), nullptr); };
    for (int it = 1; it <= w.nt; it++) {
      w.times.push_back(meteo_time_seconds(lines[i], trefstr));
      w.xe.push_back(eye(lines[i + 1]));
      w.ye.push_back(eye(lines[i + 2]));
      i += 4;
      std::vector<float>* qs[4] = {&vmag, &vdir, &pdrp, &w.prcp};
      for (int q = 0; q < w.nquant; q++)
        for (int n = 1; n <= w.nrows; n++) {
          std::istringstream ls(lines[i++]);
          for (int m = 1; m <= w.ncols; m++) ls >> (*qs[q])[w.at(it, n, m)];
        }
    }
    // sfincs_meteo.f90:65-93: absolute pressure, ring and sector widths, wind components
    w.pabs.resize(pdrp.size());
    for (size_t k = 0; k < pdrp.size(); k++) w.pabs[k] = gapres - pdrp[k];
    w.drad = w.radius / (float)w.nrows;
    w.dphi = 2.0f * pi / (float)w.ncols;
    w.wu.resize(vmag.size());
    w.wv.resize(vmag.size());
    for (size_t k = 0; k < vmag.size(); k++) {
      w.wu[k] = vmag[k] * std::cos(pi * (270.0f - vdir[k]) / 180.0f);
      w.wv[k] = vmag[k] * std::sin(pi * (270.0f - vdir[k]) / 180.0f);
    }
    spw_precip = w.nquant == 4 && use_spw_precip;
  }

  // update_spiderweb_data: sfincs_meteo.f90:450-800 (projected grids, no wave
  // age, no wind reduction). core: the core's arctangent instead of libm's.
  void update_spiderweb_data(bool core) {
    const SpwData& w = spw;
    for (int itw = 1; itw <= 2; itw++) {
      const float meteo_t = itw == 1 ? meteo_t0 : meteo_t1;
      int itw0 = 1, itw1 = 1;
      float twfac = 1.0f, tspinup_fac = 1.0f;
      if (meteo_t < w.times[0]) {
        tspinup_fac = std::max(1.0f - (w.times[0] - meteo_t) / 21600.0f, 0.0f);
      } else if (meteo_t > w.times[w.nt - 1]) {
        itw0 = itw1 = w.nt;
        tspinup_fac = std::max(1.0f - (meteo_t - w.times[w.nt - 1]) / 21600.0f, 0.0f);
      } else {
        for (int it = 1; it <= w.nt; it++)
          if (w.times[it - 1] <= meteo_t) itw0 = it;
        itw1 = std::min(itw0 + 1, w.nt);
        twfac = (meteo_t - w.times[itw0 - 1]) / std::max(w.times[itw1 - 1] - w.times[itw0 - 1], 1.0e-6f);
      }
      const float xe01 = w.xe[itw0 - 1] * (1.0f - twfac) + w.xe[itw1 - 1] * twfac;
      const float ye01 = w.ye[itw0 - 1] * (1.0f - twfac) + w.ye[itw1 - 1] * twfac;
      auto v01 = [&](const std::vector<float>& v, int irow, int icol) {
        return v[w.at(itw0, irow, icol)] * (1.0f - twfac) + v[w.at(itw1, irow, icol)] * twfac;
      };
      F1<float>& tu = itw == 1 ? tauwu0 : tauwu1;
      F1<float>& tv = itw == 1 ? tauwv0 : tauwv1;
      F1<float>& pa = itw == 1 ? patm0 : patm1;
      F1<float>& pr = itw == 1 ? prcp0 : prcp1;
      for (long nm = 1; nm <= np; nm++) {
        const float x = z_xz(nm), y = z_yz(nm);
        const float dxe = x - xe01, dye = y - ye01;
        const float dstspw = std::sqrt(dxe * dxe + dye * dye);
        if (amufile.substr(0, 4) == "none") {
          tu(nm) = 0.0f;
          tv(nm) = 0.0f;
        }
        if (patmos && ampfile.substr(0, 4) == "none") pa(nm) = gapres;
        if (precip && spw_precip && amprfile.substr(0, 4) == "none") pr(nm) = 0.0f;
        if (dstspw > w.radius) continue;
        int idstspw = std::max((int)(dstspw / w.drad), 1);
        const int ind1[4] = {idstspw, idstspw, idstspw + 1, idstspw + 1};
        if (ind1[2] > w.nrows) continue;
        const float dj1 = std::max((dstspw - w.drad * (float)idstspw) / w.drad, 0.0f);
        float phispw = 0.5f * pi - (core ? core_atan2(dye, dxe) : std::atan2(dye, dxe));
        const float tp = 2.0f * pi;
        phispw = phispw - std::floor(phispw / tp) * tp;  // modulo(phispw, 2 pi)
        const int iphispw = std::min((int)(phispw / w.dphi) + 1, w.ncols);
        int ind2[4] = {iphispw, iphispw + 1, iphispw + 1, iphispw};
        if (ind2[1] > w.ncols) ind2[1] = 1;
        if (ind2[2] > w.ncols) ind2[2] = 1;
        const float di1 = (phispw - w.dphi * (float)(iphispw - 1)) / w.dphi;
        const float f[4] = {(1.0f - di1) * (1.0f - dj1), di1 * (1.0f - dj1), di1 * dj1, (1.0f - di1) * dj1};
        float wup = 0.0f, wvp = 0.0f, prp = 0.0f, pcp = 0.0f;
        for (int ip = 0; ip < 4; ip++) {
          wup = wup + f[ip] * v01(w.wu, ind1[ip], ind2[ip]);
          wvp = wvp + f[ip] * v01(w.wv, ind1[ip], ind2[ip]);
          if (patmos) pcp = pcp + f[ip] * v01(w.pabs, ind1[ip], ind2[ip]);
          if (precip && spw_precip) prp = prp + f[ip] * v01(w.prcp, ind1[ip], ind2[ip]);
        }
        const float vmag = std::sqrt(wup * wup + wvp * wvp);
        const float cd = cdval(std::min(std::max((long)(vmag * 10.0f) + 1, 1L), 1000L));
        float merge_frac = 1.0f;
        if (dstspw > spw_merge_frac * w.radius)
          merge_frac = (1.0f / (1.0f - std::min(spw_merge_frac, 0.999f))) * (w.radius - dstspw) / w.radius;
        merge_frac = merge_frac * tspinup_fac;
        tu(nm) = (1.0f - merge_frac) * tu(nm) + merge_frac * vmag * (cosrot * wup + sinrot * wvp) * rhoa * cd / rhow;
        tv(nm) = (1.0f - merge_frac) * tv(nm) + merge_frac * vmag * (-sinrot * wup + cosrot * wvp) * rhoa * cd / rhow;
        if (patmos) pa(nm) = (1.0f - merge_frac) * pa(nm) + merge_frac * pcp;
        if (precip && spw_precip) pr(nm) = (1.0f - merge_frac) * pr(nm) + merge_frac * prp / (float)(1000 * 3600);
      }
    }
  }

  void read_meteo_data() {
    // spiderweb first (sfincs_meteo.f90:35-98), factors below (:330-412)
    if (spwfile.substr(0, 4) != "none") {
      read_spw(spwfile);
      if (factor_wind != 1.0f)
        for (size_t k = 0; k < spw.wu.size(); k++) {
          spw.wu[k] = factor_wind * spw.wu[k];
          spw.wv[k] = factor_wind * spw.wv[k];
        }
      if (factor_pres != 1.0f)
        for (auto& x : spw.pabs) x = gapres - factor_pres * (gapres - x);
      if (spw_precip && factor_prcp != 1.0f)
        for (auto& x : spw.prcp) x = factor_prcp * x;
      if (factor_spw_size != 1.0f) {
        spw.radius = factor_spw_size * spw.radius;
        spw.drad = spw.radius / (float)spw.nrows;
      }
    }
    // gridded fields (sfincs_meteo.f90:146-245) with the enhancement factors (:330-380)
    if (amufile.substr(0, 4) != "none") {
      read_am_file(amufile, amuv, 0);
      read_am_file(amvfile, amuv, 1);
      if (factor_wind != 1.0f)
        for (int q = 0; q < 2; q++)
          for (auto& x : amuv.v[q]) x = factor_wind * x;
    }
    if (amprfile.substr(0, 4) != "none") {
      read_am_file(amprfile, ampr, 0);
      if (factor_prcp != 1.0f)
        for (auto& x : ampr.v[0]) x = factor_prcp * x;
    }
    if (ampfile.substr(0, 4) != "none") {
      read_am_file(ampfile, amp, 0);
      if (factor_pres != 1.0f)
        for (auto& x : amp.v[0]) x = gapres - factor_pres * (gapres - x);
    }
    if (wndfile.substr(0, 4) != "none") {
      auto tb = read_ascii_table(path(wndfile));
      ntwnd = (long)tb.size();
      itwndlast = 1;
      twnd.alloc(ntwnd);
      wndmag.alloc(ntwnd);
      wnddir.alloc(ntwnd);
      for (long it = 1; it <= ntwnd; it++) {
        twnd(it) = (float)tb[it - 1][0];
        wndmag(it) = (float)tb[it - 1][1];
        wnddir(it) = (float)tb[it - 1][2];
        wnddir(it) = pi * (270.0f - wnddir(it)) / 180.0f - rotation;
      }
    }
    if (prcpfile.substr(0, 4) != "none") {
      auto tb = read_ascii_table(path(prcpfile));
      ntprcp = (long)tb.size();
      itprcplast = 1;
      tprcpt.alloc(ntprcp);
      tprcpv.alloc(ntprcp);
      for (long it = 1; it <= ntprcp; it++) {
        tprcpt(it) = (float)tb[it - 1][0];
        tprcpv(it) = (float)tb[it - 1][1];
      }
    }
    float cd_wnd[3] = {0.0f, 28.0f, 50.0f}, cd_val[3] = {0.0010f, 0.0025f, 0.0015f};
    int cd_nr = 3;
    cdval.alloc(1000);
    for (int iw = 1; iw <= 1000; iw++) {
      float wnd = (float)iw * 0.1f;
      for (int icd = 1; icd <= cd_nr - 1; icd++) {
        cdval(iw) = cd_val[icd - 1];
        if (wnd >= cd_wnd[icd - 1] && wnd < cd_wnd[icd]) {
          cdval(iw) = cd_val[icd - 1] +
                      (wnd - cd_wnd[icd - 1]) * (cd_val[icd] - cd_val[icd - 1]) / (cd_wnd[icd] - cd_wnd[icd - 1]);
          break;
        } else if (wnd >= cd_wnd[cd_nr - 1]) {
          cdval(iw) = cd_val[cd_nr - 1];
          break;
        }
      }
    }
  }

  // read_discharges (src/dis branch): sfincs_discharges.f90:8-324
  // read_discharges: sfincs_discharges.f90:8-320 (point sources, then drainage
  // structures, whose intake and outfall follow the sources in nmindsrc/qtsrc)
  void read_discharges() {
    nsrc = 0;
    ntsrc = 0;
    itsrclast = 1;
    ndrn = 0;
    std::vector<std::vector<double>> xy, tb;
    std::vector<std::string> drn_lines;
    if (srcfile.substr(0, 4) != "none") {
      xy = read_ascii_table(path(srcfile));
      nsrc = (long)xy.size();
      tb = read_ascii_table(path(disfile));
      ntsrc = (long)tb.size();
    }
    if (drnfile.substr(0, 4) != "none") {
      std::ifstream fin(path(drnfile));
      if (!fin) throw std::runtime_error("oracle: cannot open " + drnfile);
      for (std::string l; std::getline(fin, l);) {
        for (char& ch : l)
          if (ch == ',' || ch == '\t' || ch == '\r') ch = ' ';
        if (l.find_first_not_of(' ') != std::string::npos) drn_lines.push_back(l);
      }
      ndrn = (long)drn_lines.size();
    }
    nsrcdrn = nsrc + 2 * ndrn;
    if (nsrcdrn > 0) {
      nmindsrc.alloc(nsrcdrn);
      qtsrc.alloc(nsrcdrn);
    }
    if (nsrc > 0) {
      tsrc.alloc(ntsrc);
      qsrc.alloc(nsrc, ntsrc);
      for (long it = 1; it <= ntsrc; it++) {
        tsrc(it) = (float)tb[it - 1][0];
        for (long is = 1; is <= nsrc; is++) qsrc(is, it) = (float)tb[it - 1][is];
      }
      for (long is = 1; is <= nsrc; is++) {
        long nmq = find_quadtree_cell((float)xy[is - 1][0], (float)xy[is - 1][1]);
        nmindsrc(is) = nmq > 0 ? index_sfincs_in_quadtree(nmq) : 0;
        if (nmindsrc(is) == 0) throw std::runtime_error("oracle: source point outside the active mesh");
      }
    }
    if (ndrn > 0) {
      drainage_type.alloc(ndrn);
      drainage_params.alloc(ndrn, 6);
      drainage_status.alloc(ndrn, 1);             // open
      drainage_distance.alloc(ndrn);
      drainage_fraction_open.alloc(ndrn, 1.0f);  // fully open
      for (long idrn = 1; idrn <= ndrn; idrn++) {
        std::istringstream ls(drn_lines[idrn - 1]);
        float xsnk, ysnk, xsrc, ysrc;
        int type = 0;
        ls >> xsnk >> ysnk >> xsrc >> ysrc >> type;
        int npars = (type >= 1 && type <= 3) ? 1 : ((type == 4 || type == 5) ? 6 : 0);
        if (npars == 0) throw std::runtime_error("oracle: drainage type not recognized");
        drainage_type(idrn) = (int8_t)type;
        for (int k = 1; k <= npars; k++)
          if (!(ls >> drainage_params(idrn, k))) throw std::runtime_error("oracle: drainage parameters missing");
        long j = nsrc + idrn * 2 - 1;
        long nmq = find_quadtree_cell(xsnk, ysnk);
        if (nmq > 0) nmindsrc(j) = index_sfincs_in_quadtree(nmq);
        j = nsrc + idrn * 2;
        nmq = find_quadtree_cell(xsrc, ysrc);
        if (nmq > 0) nmindsrc(j) = index_sfincs_in_quadtree(nmq);
        long a = nmindsrc(nsrc + idrn * 2 - 1), b = nmindsrc(nsrc + idrn * 2);
        if (a == 0 || b == 0) throw std::runtime_error("oracle: drainage point outside the active mesh");
        float xsnk_tmp = z_xz(a), ysnk_tmp = z_yz(a), xsrc_tmp = z_xz(b), ysrc_tmp = z_yz(b);
        drainage_distance(idrn) =
            std::sqrt((xsrc_tmp - xsnk_tmp) * (xsrc_tmp - xsnk_tmp) + (ysrc_tmp - ysnk_tmp) * (ysrc_tmp - ysnk_tmp));
      }
    }
  }

  // find_quadtree_cell: sfincs_quadtree.F90:764-820
  long find_quadtree_cell(float x, float y) {
    float xt = qt_cosrot * (x - qt_x0) + qt_sinrot * (y - qt_y0);
    float yt = -qt_sinrot * (x - qt_x0) + qt_cosrot * (y - qt_y0);
    for (int iref = qt_nlev; iref >= 1; iref--) {
      long n = (long)(yt / qt_dyr(iref)) + 1;
      long m = (long)(xt / qt_dxr(iref)) + 1;
      long idx = find_qt_by_index(n, m, iref);
      if (idx > 0 && qt_level(idx) == iref) return idx;
    }
    return 0;
  }

  void initialize(const std::string& d, bool bmi) {
    dir = d;
    read_sfincs_input();
    use_qext = bmi;
    read_meteo_data();
    initialize_processes();
    initialize_mesh();
    initialize_bathymetry();
    initialize_boundaries();
    initialize_roughness();
    initialize_infiltration();
    initialize_hydro();
    fill_h73_tables();
    if (qt_nlev == 1) use_quadtree = false;  // sfincs_domain.f90:42-50
    set_advection_mask();
    read_structures();  // sfincs_lib.f90:156, after initialize_domain
    read_crs_file();
    read_rug_file();
    read_boundary_data();
    find_boundary_indices();
    read_discharges();
    t = t0;  // sfincs_lib.f90:279-292
    dt = 1.0e-6f;
    min_dt = 1.0e-6f;
    dtavg = 0.0f;
    nt = 0;
  }

  // fill_h73_tables: sfincs_data.f90:858-881.  x73(j, k) = hh**2 * hh**(1.0/3.0),
  // hh = 0.001 * j * 10.0**(k - 6); stored 1-based at (k - 1) * 1000 + j.
  void fill_h73_tables() {
    if (!h73table) return;
    x73.alloc(10000);
    for (int k = 1; k <= 10; k++) {
      T p10 = (T)1;
      for (int i = 0; i < std::abs(k - 6); i++) p10 = p10 * (T)10;
      if (k < 6) p10 = (T)1 / p10;
      for (int j = 1; j <= 1000; j++) {
        T hh = (T)0.001f * (T)j * p10;
        x73((long)(k - 1) * 1000 + j) = hh * hh * std::pow(hh, (T)(1.0f / 3.0f));
      }
    }
  }
  // power7over3: sfincs_momentum.f90:787-820 (row clamped to 1..1000)
  T power7over3(T hu) {
    static const float lim[10] = {0.00001f, 0.0001f, 0.001f, 0.01f, 0.1f, 1.0f, 10.0f, 100.0f, 1000.0f, 10000.0f};
    static const float scl[10] = {1e8f, 1e7f, 1e6f, 1e5f, 1e4f, 1e3f, 100.0f, 10.0f, 1.0f, 0.1f};
    for (int k = 1; k <= 10; k++) {
      if (hu < (T)lim[k - 1]) {
        long j = std::min(std::max((long)((T)scl[k - 1] * hu), 1L), 1000L);
        return x73((long)(k - 1) * 1000 + j);
      }
    }
    return (T)std::pow((T)10000, (T)(7.0f / 3.0f));
  }

  // ============================================================ time step
  // update_meteo_forcing (time-series part): sfincs_meteo.f90:1246-1558
  // update_meteo_fields: sfincs_meteo.f90:1561-1624 (ASCII gridded meteo)
  void update_meteo_fields() {
    if (amufile.substr(0, 4) != "none") update_am_window(amuv, 0);
    if (ampfile.substr(0, 4) != "none" && patmos) update_am_window(amp, 1);
    if (amprfile.substr(0, 4) != "none") update_am_window(ampr, 2);
    if (spwfile.substr(0, 4) != "none") update_spiderweb_data(std::is_same<TZ, float>::value);
  }

  void update_meteo_forcing(double tt, float dtt) {
    if (meteo3d) {  // :1264-1417
      const float twfact = (float)((tt - (double)meteo_t0) / (double)(meteo_t1 - meteo_t0));
      const float onemintwfact = 1.0f - twfact;
      for (long nm = 1; nm <= np; nm++) {
        if (wind) {
          tauwu(nm) = tauwu0(nm) * onemintwfact + tauwu1(nm) * twfact;
          tauwv(nm) = tauwv0(nm) * onemintwfact + tauwv1(nm) * twfact;
        }
        if (patmos) patm(nm) = patm0(nm) * onemintwfact + patm1(nm) * twfact;
        if (precip) {
          prcp(nm) = prcp0(nm) * onemintwfact + prcp1(nm) * twfact;
          if (prcp(nm) < 0.0f) {  // no negative rain on a dry cell
            if (subgrid ? z_volume(nm) <= 0.0 : (double)zs(nm) <= (double)zb(nm)) prcp(nm) = 0.0f;
          }
          netprcp(nm) = prcp(nm);
          if (store_cumulative_precipitation) cumprcp(nm) = cumprcp(nm) + prcp(nm) * dtt;
        }
      }
      if (tt < (double)(tspinup - 1.0e-3f) && spinup_meteo) {  // :1349-1398
        const float smfac = (float)((tt - (double)t0) / (double)(tspinup - t0));
        const float oneminsmfac = 1.0f - smfac;
        for (long nm = 1; nm <= np; nm++) {
          if (wind) {
            tauwu(nm) = tauwu(nm) * smfac;
            tauwv(nm) = tauwv(nm) * smfac;
          }
          if (patmos) patm(nm) = patm(nm) * smfac + gapres * oneminsmfac;
          if (precip) {
            netprcp(nm) = netprcp(nm) * smfac;
            if (netprcp(nm) < 0.0f) {
              if (subgrid ? z_volume(nm) <= 0.0 : (double)zs(nm) <= (double)zb(nm)) netprcp(nm) = 0.0f;
            }
          }
        }
      }
      if (patmos && pavbnd > 0.0f)  // :1400-1417
        for (long ib = 1; ib <= ngbnd; ib++) patmb(ib) = patm(nmindbnd(ib));
    }
    if (wind && wndfile.substr(0, 4) != "none") {  // update_wind_forcing_from_timeseries :1445-1508
      for (long itw = itwndlast; itw <= ntwnd; itw++) {
        if ((double)twnd(itw) > tt) {
          long i0 = std::max(itw - 1, 1L);  // out-of-range guard: series must cover t
          float twfac = (float)((tt - (double)twnd(i0)) / (double)(twnd(itw) - twnd(i0)));
          float vmag = wndmag(i0) * (1.0f - twfac) + wndmag(itw) * twfac;
          float twopi = 2.0f * pi;
          float dr0 = std::fmod(wnddir(i0), twopi);
          if (dr0 < 0) dr0 += twopi;
          float dr1 = std::fmod(wnddir(itw), twopi);
          if (dr1 < 0) dr1 += twopi;
          if (dr1 > dr0 + pi)
            dr0 = dr0 + 2.0f * pi;
          else if (dr0 > dr1 + pi)
            dr1 = dr1 + 2.0f * pi;
          float vdir = dr0 * (1.0f - twfac) + dr1 * twfac;
          float cd = cdval((long)(vmag * 10.0f) + 1);
          double twu = (double)(vmag * vmag * std::cos(vdir) * rhoa * cd / rhow);
          double twv = (double)(vmag * vmag * std::sin(vdir) * rhoa * cd / rhow);
          for (long nm = 1; nm <= np; nm++) {
            tauwu(nm) = (float)twu;
            tauwv(nm) = (float)twv;
          }
          itwndlast = itw - 1 >= 1 ? itw - 1 : 1;
          break;
        }
      }
    }
    if (precip && prcpfile.substr(0, 4) != "none") {  // update_precipitation_from_timeseries :1510-1558
      long itp;
      for (itp = itprcplast; itp <= ntprcp; itp++)
        if ((double)tprcpt(itp) > tt) break;
      itp = std::max(std::min(itp, ntprcp), 1L);
      long i0 = std::max(itp - 1, 1L);  // out-of-range guard: series must cover t
      float twfac = (float)((tt - (double)tprcpt(i0)) / (double)(tprcpt(itp) - tprcpt(i0)));
      if (i0 == itp) twfac = 0.0f;
      float ptmp = (tprcpv(i0) * (1.0f - twfac) + tprcpv(itp) * twfac) / (float)(1000 * 3600);
      for (long nm = 1; nm <= np; nm++) {
        prcp(nm) = ptmp;
        netprcp(nm) = ptmp;
        if (store_cumulative_precipitation) cumprcp(nm) = cumprcp(nm) + ptmp * dtt;
      }
      itprcplast = itp - 1 >= 1 ? itp - 1 : 1;
    }
  }

  // update_infiltration_map: sfincs_infiltration.f90:609-1039
  void update_infiltration_map(float dtt) {
    constexpr bool CORE = std::is_same<TZ, float>::value;
    // gai reads GA_head(np) * GA_sigma(np) for every cell (:858); in the
    // reference's serial order every cell sees the last cell's value from
    // before this update
    const float ga_hs = inftype == "gai" ? GA_head(np) * GA_sigma(np) : 0.0f;
    for (long nm = 1; nm <= np; nm++) {
      if (inftype == "con" || inftype == "c2d") {  // :632-676
        qinfmap(nm) = qinffield(nm);
        if (subgrid) {
          if (z_volume(nm) <= 0.0) qinfmap(nm) = 0.0f;
        } else {
          if (zs(nm) <= zb(nm)) qinfmap(nm) = 0.0f;
        }
      } else if (inftype == "cna") {  // :678-723
        if (cumprcp(nm) > sfacinf * qinffield(nm)) {
          float a = cumprcp(nm) - sfacinf * qinffield(nm);
          float Qq = a * a / (cumprcp(nm) + (1.0f - sfacinf) * qinffield(nm));
          float I = cumprcp(nm) - Qq;
          qinfmap(nm) = (I - cuminf(nm)) / dtt;
        } else {
          qinfmap(nm) = prcp(nm);
        }
      } else if (inftype == "cnb") {  // :724-829
        if (prcp(nm) > 0.0f) {
          if (scs_rain(nm) != 1) {
            scs_P1(nm) = 0.0f;
            scs_F1(nm) = 0.0f;
            scs_S1(nm) = scs_Se(nm);
            scs_rain(nm) = 1;
          }
          scs_P1(nm) = scs_P1(nm) + prcp(nm) * dtt;
          if (scs_P1(nm) > sfacinf * scs_S1(nm)) {
            float a = scs_P1(nm) - sfacinf * scs_S1(nm);
            float Qq = a * a / (scs_P1(nm) + (1.0f - sfacinf) * scs_S1(nm));
            float I = scs_P1(nm) - Qq;
            qinfmap(nm) = (I - scs_F1(nm)) / dtt;
            scs_F1(nm) = I;
          } else {
            scs_F1(nm) = scs_P1(nm);
            qinfmap(nm) = prcp(nm);
          }
          scs_Se(nm) = std::max(scs_Se(nm) - qinfmap(nm) * dtt, 0.0f);
          qinfmap(nm) = std::max(qinfmap(nm), 0.0f);
        } else {
          if (scs_rain(nm) == 1) {
            scs_rain(nm) = 0;
            qinfmap(nm) = 0.0f;
            rain_T1(nm) = 0.0f;
          }
          rain_T1(nm) = rain_T1(nm) + dtt / 3600.0f;
          if (rain_T1(nm) > 0.06f / inf_kr(nm)) {
            scs_Se(nm) = scs_Se(nm) + inf_kr(nm) * qinffield(nm) * dtt / 3600.0f;
            scs_Se(nm) = std::min(scs_Se(nm), qinffield(nm));
          }
        }
      } else if (inftype == "gai") {  // :830-912; qinfmap keeps its last value while it does not rain
        if (prcp(nm) > 0.0f) {
          if (prcp(nm) < ksfield(nm)) {
            qinfmap(nm) = prcp(nm);
          } else {
            qinfmap(nm) = ksfield(nm) * (1.0f + ga_hs / GA_F(nm));
            qinfmap(nm) = std::fmax(std::fmin(qinfmap(nm), prcp(nm)), 0.0f);
          }
          GA_sigma(nm) = std::max(GA_sigma(nm) - qinfmap(nm) * dtt / GA_Lu(nm), 0.0f);
          GA_F(nm) = GA_F(nm) + qinfmap(nm) * dtt;
          rain_T1(nm) = 0.0f;
        } else {
          rain_T1(nm) = rain_T1(nm) + dtt / 3600.0f;
          if (rain_T1(nm) > 0.06f / inf_kr(nm)) {
            GA_sigma(nm) = GA_sigma(nm) + inf_kr(nm) * GA_sigma_max(nm) * dtt / 3600.0f;
            GA_sigma(nm) = std::min(GA_sigma(nm), GA_sigma_max(nm));
            GA_F(nm) = std::max(GA_F(nm) - inf_kr(nm) * GA_sigma_max(nm) * dtt / 3600.0f * GA_Lu(nm), 0.0f);
          }
        }
      } else if (inftype == "hor") {  // :914-1033
        float hh_local = subgrid ? (float)(z_volume(nm) / (double)area_of(nm))
                                 : (float)((double)zs(nm) - (double)zb(nm));
        if (hh_local > 0.0f || prcp(nm) > 0.0f) {
          if (rain_T1(nm) > 0.0f)
            rain_T1(nm) = 0.0f;
          else
            rain_T1(nm) = rain_T1(nm) - dtt;
          float x = horton_kd(nm) * rain_T1(nm) / 3600.0f;
          float I = CORE ? core_exp(x) : std::exp(x);
          if (I < 0.01f) {
            I = 0.0f;
            rain_T1(nm) = rain_T1(nm) + dtt;
            qinfmap(nm) = horton_fc(nm) / 3600.0f / 1000.0f;
          } else {
            qinfmap(nm) = (horton_fc(nm) + (horton_f0(nm) - horton_fc(nm)) * I) / 3600.0f / 1000.0f;
          }
          float Qq = hh_local > 0.0f ? prcp(nm) * dtt + hh_local : prcp(nm) * dtt;
          I = qinfmap(nm) * dtt;
          if (I > Qq) qinfmap(nm) = qinfmap(nm) * Qq / I;
        } else {
          rain_T1(nm) = rain_T1(nm) + dtt / horton_kr_kd;
          qinfmap(nm) = 0.0f;
        }
      }
      netprcp(nm) = netprcp(nm) - qinfmap(nm);
      if (store_cumulative_precipitation) cuminf(nm) = cuminf(nm) + qinfmap(nm) * dtt;
    }
  }

  // The bca file (sfincs_boundaries.f90:289-450): two passes over the lines,
  // cleaned as clean_line (:1242-1252) does; then update_nodal_factors at the
  // date of tref (astro.f90:5-96, time_to_vector sfincs_date.f90:329-364,
  // datumi astro.f90:646-748).  Inputs the reference would index outside its
  // arrays with are refused.
  void read_bca() {
    std::ifstream in(path(bcafile));
    if (!in) throw std::runtime_error("oracle: cannot open " + bcafile);
    std::vector<std::string> lines;
    for (std::string l; std::getline(in, l);) {
      const size_t cr = l.find('\r');
      if (cr != std::string::npos) l = l.substr(0, cr);
      const size_t a = l.find_first_not_of(' ');
      l = a == std::string::npos ? std::string() : l.substr(a);
      while (!l.empty() && (l.back() == ' ' || l.back() == '\t')) l.pop_back();
      lines.push_back(l);
    }
    auto meta = [](const std::string& l) {
      for (const char* k : {"Quantity", "Unit", "Name", "Function", "quantity", "unit", "name", "function"})
        if (l.find(k) != std::string::npos) return true;
      return false;
    };
    auto data = [](const std::string& l, std::string& cname, float& a, float& p) {
      std::string t = l;
      for (char& c : t)
        if (c == ',' || c == '\t') c = ' ';
      std::istringstream is(t);
      std::string sa, sp;
      if (!(is >> cname >> sa >> sp)) return false;
      char* e;
      a = std::strtof(sa.c_str(), &e);
      if (e == sa.c_str() || *e) return false;
      p = std::strtof(sp.c_str(), &e);
      if (e == sp.c_str() || *e) return false;
      return true;
    };
    long n_sets = 0, n_components = 0;
    bool has_a0 = false;
    for (const auto& l : lines) {
      std::string cname;
      float a, p;
      if (l == "[forcing]" || l == "[Forcing]") n_sets++;
      else if (meta(l)) continue;
      else if (data(l, cname, a, p)) {
        if (n_sets == 0) throw std::runtime_error("oracle: bca data before the first [forcing]");
        if (n_sets == 1) {
          n_components++;
          if (n_components == 1 && (cname.compare(0, 2, "a0") == 0 || cname.compare(0, 2, "A0") == 0)) has_a0 = true;
        }
      }
    }
    if (n_sets != nbnd) throw std::runtime_error("oracle: bca sets do not match the bnd points");
    if (!has_a0) n_components++;
    const long nc = n_components;
    nr_tidal_components = nc;
    tidal_component_names.assign(nc, "");
    tidal_amp.assign((size_t)nc * nbnd, 0.0);
    tidal_phase.assign((size_t)nc * nbnd, 0.0);
    long current_set = 0, current_component = 0;
    for (const auto& l : lines) {
      std::string cname;
      float a, p;
      if (l == "[forcing]" || l == "[Forcing]") {
        current_set++;
        current_component = 0;
        if (!has_a0) {
          current_component = 1;
          tidal_component_names[0] = "A0";
        }
      } else if (meta(l)) {
        continue;
      } else if (data(l, cname, a, p)) {
        current_component++;
        if (current_component > nc) throw std::runtime_error("oracle: bca set longer than the first");
        tidal_component_names[current_component - 1] = cname;
        tidal_amp[(size_t)(current_set - 1) * nc + current_component - 1] = (double)a;
        tidal_phase[(size_t)(current_set - 1) * nc + current_component - 1] = (double)p;
      }
    }
    // time_to_vector(0, tref): the time of day through real*4 fractions
    const int yyyy = std::atoi(trefstr.substr(0, 4).c_str()), mm = std::atoi(trefstr.substr(4, 2).c_str()),
              dd = std::atoi(trefstr.substr(6, 2).c_str()), hh = std::atoi(trefstr.substr(9, 2).c_str()),
              mn = std::atoi(trefstr.substr(11, 2).c_str()), ss = std::atoi(trefstr.substr(13, 2).c_str());
    const float ref_fraction = (float)hh / 24 + (float)mn / 1440 + (float)ss / 86400;
    const float sec_add = (float)((double)(ref_fraction * 86400) + 0.0);
    const int ndays_add = (int)(sec_add / 86400);
    if (ndays_add != 0) throw std::runtime_error("oracle: tref time of day out of range");
    const float secs_time = sec_add - (float)ndays_add * 86400.0f;
    const int h = (int)(secs_time / 3600);
    const int mi = (int)((secs_time - (float)(h * 3600)) / 60);
    const int se = (int)(secs_time - (float)(h * 3600) - (float)(mi * 60));
    // datumi: hours into the year
    double rmd[13] = {0, 0, 31, 59, 90, 120, 151, 181, 212, 243, 273, 304, 334};
    if (yyyy % 4 == 0 && (yyyy % 100 != 0 || yyyy % 400 == 0))
      for (int i = 3; i <= 12; i++) rmd[i] += 1.0;
    const double thours = rmd[mm] * 24.0 + (double)(float)(dd - 1) * 24.0 + (double)(float)h +
                          (double)(float)mi / 60.0 + (double)(float)se / 3600.0;
    double v[16] = {0}, f[26] = {0};
    astro_hulpgr(yyyy, thours, v, f);
    const double pi = (double)(4.0f * std::atan(1.0f));  // 4 * atan(1.0): single precision
    tidal_component_frequency.assign(nc, 0.0);         // A0: left unset by the reference, 0 here
    for (long k = 2; k <= nc; k++) {
      std::string nm = tidal_component_names[k - 1];
      if (nm == "EPS2") nm = "EPSILON2";
      if (nm == "LA2") nm = "LABDA2";
      if (nm == "MTM") nm = "MFM";
      double w, v0u, fr;
      if (!astro_bewvuf(nm, v, f, w, v0u, fr)) throw std::runtime_error("oracle: constituent " + nm + " not carried");
      tidal_component_frequency[k - 1] = w / 3600;
      for (long n = 1; n <= nbnd; n++) {
        double& A = tidal_amp[(size_t)(n - 1) * nc + k - 1];
        double& P = tidal_phase[(size_t)(n - 1) * nc + k - 1];
        A = A * fr;
        P = (pi / 180) * P - v0u;
        double r = std::fmod(P, 2 * pi);  // MODULO(P, 2 pi)
        if (r != 0.0 && r < 0.0) r = r + 2 * pi;
        P = r;
      }
    }
  }

  // update_boundary_points: sfincs_boundaries.f90:682-758
  void update_boundary_points(double tt) {
    if (nbnd == 0) return;
    long itb0 = 1, itb1 = 1;
    float tb = 0.0f;
    if ((double)t_bnd(1) > (tt - 1.0e-3)) {
      itb0 = 1;
      itb1 = 1;
      tb = t_bnd(itb0);
    } else if ((double)t_bnd(ntbnd) < (tt + 1.0e-3)) {
      itb0 = ntbnd;
      itb1 = ntbnd;
      tb = t_bnd(itb0);
    } else {
      for (long itb = itbndlast; itb <= ntbnd; itb++) {
        if ((double)t_bnd(itb) > (tt + 1.0e-6)) {
          itb0 = itb - 1;
          itb1 = itb;
          tb = (float)tt;
          itbndlast = itb - 1;
          break;
        }
      }
    }
    float tbfac = (tb - t_bnd(itb0)) / std::max(t_bnd(itb1) - t_bnd(itb0), 1.0e-6f);
    const bool core = std::is_same<TZ, float>::value;
    for (long ib = 1; ib <= nbnd; ib++) {
      float zstb = zs_bnd(ib, itb0) + (zs_bnd(ib, itb1) - zs_bnd(ib, itb0)) * tbfac;
      const long nc = nr_tidal_components;
      for (long ic = 1; ic <= nc; ic++) {  // astronomic tides (:736-744)
        const double arg = tidal_component_frequency[ic - 1] * tt - tidal_phase[(size_t)(ib - 1) * nc + ic - 1];
        zstb = (float)((double)zstb + tidal_amp[(size_t)(ib - 1) * nc + ic - 1] * (core ? core_cos(arg) : std::cos(arg)));
      }
      zst_bnd(ib) = zstb;
    }
  }

  // update_boundary_conditions: sfincs_boundaries.f90:761-921
  void update_boundary_conditions(double tt) {
    for (long ib = 1; ib <= ngbnd; ib++) {
      long nmb = nmindbnd(ib);
      if (kcs(nmb) == 2) {
        double zst;
        if (nbnd > 1)
          zst = (double)(zst_bnd(ind1_bnd_gbp(ib)) * fac_bnd_gbp(ib) +
                         zst_bnd(ind2_bnd_gbp(ib)) * (1.0f - fac_bnd_gbp(ib)));
        else
          zst = (double)zst_bnd(1);
        if (patmos && pavbnd > 1.0f)  // barometric correction (sfincs_boundaries.f90:820-826)
          zst = zst + (double)((pavbnd - patmb(ib)) / (rhow * 9.81f));
        float zsetup = 0.0f, zig = 0.0f;
        if (tt < (double)(tspinup - 1.0e-3f)) {
          float smfac = (float)(1.0 - (tt - (double)t0) / (double)(tspinup - t0));
          float zs0act = (float)(zst + (double)zsetup);
          zsb0(ib) = zini * smfac + zs0act * (1.0f - smfac);
          zs0act = (float)(zst + (double)zsetup + (double)zig);
          zsb(ib) = zini * smfac + zs0act * (1.0f - smfac);
        } else {
          zsb0(ib) = (float)(zst + (double)zsetup);
          zsb(ib) = (float)(zst + (double)zsetup + (double)zig);
        }
        if (subgrid) {
          zsb0(ib) = std::max(zsb0(ib), sg_z_zmin(nmb));
          zsb(ib) = std::max(zsb(ib), sg_z_zmin(nmb));
        } else {
          zsb0(ib) = std::max(zsb0(ib), zb(nmb));
          zsb(ib) = std::max(zsb(ib), zb(nmb));
        }
      } else if (kcs(nmb) == 5) {  // downstream river point (:878-902)
        long ibdr = index_bdr_gbp(ib);
        double zst = (double)zs(index_zsi_bdr(ibdr)) + (double)dzs_bdr(ibdr);
        zst = std::max(zst, subgrid ? (double)sg_z_zmin(nmb) : (double)zb(nmb));
        zsb(ib) = (float)zst;
        zsb0(ib) = (float)zst;
      } else if (kcs(nmb) == 6) {
        zs(nmb) = zs(nmi_gbp(ib));
      }
    }
  }

  // update_boundary_fluxes: sfincs_boundaries.f90:924-1122
  void update_boundary_fluxes(float dtt, double tt) {
    float factime = std::min(dtt / btfilter, 1.0f);
    float one_minus_factime = 1.0f - factime;
    float facrel = 1.0f - std::min(dtt / btrelax, 1.0f);
    long L = subgrid_nlevels;
    for (long ib = 1; ib <= nkcuv2; ib++) {
      long indb = ibkcuv2(ib);
      long nmb = nmbkcuv2(ib);
      if (kcs(nmb) == 6) continue;
      long nmi = nmikcuv2(ib);
      long ip = index_kcuv2(ib);
      float zsnmi = (float)zs(nmi);
      float zsnmb = zsb(indb);
      float zs0nmb = zsb0(indb);
      float hnmb;
      if (bndtype == 1) {
        if (subgrid) {
          float zsuv = std::max(zsnmb, zsnmi);
          float depthuv;
          if (zsuv >= sg_uv_zmax(ip) - 1.0e-4f) {
            depthuv = sg_uv_havg_zmax(ip) + zsuv;
          } else if (zsuv > sg_uv_zmin(ip)) {
            float dzuv = (sg_uv_zmax(ip) - sg_uv_zmin(ip)) / (float)(L - 1);
            long iuv = (long)((zsuv - sg_uv_zmin(ip)) / dzuv) + 1;
            float facint = (zsuv - (sg_uv_zmin(ip) + (float)(iuv - 1) * dzuv)) / dzuv;
            depthuv = sg_uv_havg(iuv, ip) + (sg_uv_havg(iuv + 1, ip) - sg_uv_havg(iuv, ip)) * facint;
          } else {
            depthuv = 0.0f;
          }
          hnmb = std::max(depthuv, huthresh);
          zsnmb = std::max(zsnmb, sg_z_zmin(nmb));
          zs0nmb = std::max(zs0nmb, sg_z_zmin(nmb));
        } else {
          hnmb = std::max(0.5f * (zsnmb + zsnmi) - zbuv(ip), huthresh);
          zsnmb = std::max(zsnmb, zb(nmb));
          zs0nmb = std::max(zs0nmb, zb(nmb));
        }
        if (hnmb < huthresh + 1.0e-6f || kcuv(ip) == 3) {
          q(ip) = (T)0;
          uv(ip) = (T)0;
          uvmean(ib) = 0.0f;
        } else {
          float sq = std::sqrt(g / hnmb);
          float ui = sq * (zsnmb - zs0nmb);
          float ub = (float)ibuvdir(ib) * (2.0f * ui - sq * (zsnmi - zs0nmb));
          float qq = ub * hnmb + uvmean(ib);
          if (subgrid) {
            if (z_volume(nmi) <= 0.0) qq = ibuvdir(ib) == 1 ? std::max(qq, 0.0f) : std::min(qq, 0.0f);
            if (zsnmb - sg_z_zmin(nmb) < huthresh) qq = ibuvdir(ib) == 1 ? std::min(qq, 0.0f) : std::max(qq, 0.0f);
          } else {
            if (zsnmi - zb(nmi) <= huthresh) qq = ibuvdir(ib) == 1 ? std::max(qq, 0.0f) : std::min(qq, 0.0f);
            if (zsnmb - zb(nmb) < huthresh) qq = ibuvdir(ib) == 1 ? std::min(qq, 0.0f) : std::max(qq, 0.0f);
          }
          q(ip) = (T)qq;
          uv(ip) = (T)std::max(std::min(qq / hnmb, 4.0f), -4.0f);
        }
        if (btfilter >= -1.0e-6f)
          uvmean(ib) = factime * (float)q(ip) + facrel * one_minus_factime * uvmean(ib);
        else
          uvmean(ib) = 0.0f;
        zs(nmb) = (TZ)zsb(indb);
        if (store_maximum_waterlevel) {
          if (store_t_zsmax && zs(nmb) > zsmax(nmb)) t_zsmax(nmb) = (float)tt;
          zsmax(nmb) = (T)std::max((double)zsmax(nmb), (double)zs(nmb));
        }
      }
    }
  }

  // update_discharges (point sources): sfincs_discharges.f90:325-368
  // update_discharges: sfincs_discharges.f90:325-659
  void update_discharges(double tt) {
    if (nsrc > 0) {
      for (long its = itsrclast; its <= ntsrc; its++) {
        if ((double)tsrc(its) > tt) {
          long i0 = std::max(its - 1, 1L);
          for (long is = 1; is <= nsrc; is++)
            qtsrc(is) = (float)((double)qsrc(is, i0) +
                                (double)(qsrc(is, its) - qsrc(is, i0)) * (tt - (double)tsrc(i0)) /
                                    (double)(tsrc(its) - tsrc(i0)));
          itsrclast = its - 1 >= 1 ? its - 1 : 1;
          break;
        }
      }
    }
    const bool core = std::is_same<TZ, float>::value;  // the core's precision: zs in FP32
    for (long idrn = 1; idrn <= ndrn; idrn++) {
      long jin = nsrc + idrn * 2 - 1, jout = nsrc + idrn * 2;
      long nmin = nmindsrc(jin), nmout = nmindsrc(jout);
      if (!(nmin > 0 && nmout > 0)) continue;
      const double zin = (double)zs(nmin), zout = (double)zs(nmout);  // zs is real*8 in the reference
      float qq = 0.0f;
      int type = drainage_type(idrn);
      if (type == 1) {  // pump
        qq = drainage_params(idrn, 1);
      } else if (type == 2 || type == 3) {  // culvert, check valve
        if (zin > zout)
          qq = (float)((double)drainage_params(idrn, 1) * std::sqrt(zin - zout));
        else
          qq = (float)((double)(-drainage_params(idrn, 1)) * std::sqrt(zout - zin));
        if (type == 3) qq = std::max(qq, 0.0f);
      } else {  // controlled gates (4: by level at the intake, 5: by time)
        float wdt = drainage_params(idrn, 1), zsill = drainage_params(idrn, 2), mng = drainage_params(idrn, 3);
        float tcls = drainage_params(idrn, 6);
        float dzds = (float)((zout - zin) / (double)drainage_distance(idrn));
        float frac = drainage_fraction_open(idrn);
        float hgate = (float)std::max(std::max(zin, zout) - (double)zsill, 0.0);
        float dfrac = dt / tcls;
        float qq0 = -qtsrc(jin) / (wdt * std::max(frac, 0.001f));
        int status = drainage_status(idrn);
        if (type == 4) {
          float zmin = drainage_params(idrn, 4), zmax = drainage_params(idrn, 5);
          if (status == 0) {
            if (zin > (double)zmin && zin < (double)zmax) status = 3;
          } else if (status == 1) {
            if (zin <= (double)zmin || zin >= (double)zmax) status = 2;
          }
        } else {
          float tclose = drainage_params(idrn, 4), topen = drainage_params(idrn, 5);
          if (status == 0) {
            if (tt >= (double)topen) status = 3;
          } else if (status == 1) {
            if (tt >= (double)tclose && tt < (double)topen) status = 2;
          }
        }
        if (status == 2) {
          frac = frac - dfrac;
          if (frac < 0.0f) {
            frac = 0.0f;
            status = 0;
          }
        } else if (status == 3) {
          frac = frac + dfrac;
          if (frac > 1.0f) {
            frac = 1.0f;
            status = 1;
          }
        }
        drainage_fraction_open(idrn) = frac;
        drainage_status(idrn) = (int8_t)status;
        // hgate**(7.0/3.0); the core's precision evaluates it as hgate**2 * cube root(hgate)
        float h73 = core ? hgate * hgate * core_cube_root(hgate) : std::pow(hgate, 7.0f / 3.0f);
        qq = (qq0 - g * hgate * dzds * dt) / (1.0f + g * (mng * mng) * dt * std::fabs(qq0) / h73);
        qq = qq * wdt * frac;
      }
      qq = 1.0f / (structure_relax / dt) * qq + (1.0f - (1.0f / (structure_relax / dt))) * -qtsrc(jin);
      if (subgrid) {
        if (qq > 0.0f)
          qq = (float)std::min((double)qq, std::max((double)z_volume(nmin), 0.0) / (double)dt);
        else
          qq = (float)std::max((double)qq, -std::max((double)z_volume(nmout), 0.0) / (double)dt);
      } else {
        if (qq > 0.0f)
          qq = (float)std::min((double)qq, std::max((zin - (double)zb(nmin)) * (double)cell_area(z_flags_iref(nmin)), 0.0) / (double)dt);
        else
          qq = (float)std::max((double)qq, -std::max((zout - (double)zb(nmout)) * (double)cell_area(z_flags_iref(nmout)), 0.0) / (double)dt);
      }
      qtsrc(jin) = -qq;
      qtsrc(jout) = qq;
    }
  }

  // compute_fluxes: sfincs_momentum.f90:9-784 (projected grids)
  void compute_fluxes(float dtt) {
    min_dt = dtmax;
    for (long ip = 1; ip <= npuv + ncuv; ip++) {
      q0(ip) = q(ip);
      uv0(ip) = uv(ip);
    }
    const T expo = (T)(1.0f / 3.0f);
    const long L = subgrid_nlevels;
    float mdt = min_dt;
    // The core-precision instantiation evaluates a few expressions as the CUDA
    // core does (one division for the table interval and one for the flux
    // update, fused multiply-adds, its own cube root); "ref" and "fp64" keep
    // the reference's expressions.
    constexpr bool CORE = std::is_same<TZ, float>::value;
#pragma omp parallel for schedule(dynamic, 256) reduction(min : mdt)
    for (long ip = 1; ip <= npuv; ip++) {
      if (!(kcuv(ip) == 1 || kcuv(ip) == 6)) continue;
      long nm = uv_index_z_nm(ip), nmu = uv_index_z_nmu(ip);
      bool iok = false;
      T zsu = (T)std::max(zs(nm), zs(nmu));
      T zmin = 0, zmax = 0;
      if (subgrid) {
        zmin = sg_uv_zmin(ip);
        zmax = sg_uv_zmax(ip);
        if (zsu > zmin + (T)huthresh) iok = true;
      } else {
        if (zsu > (T)zbuvmx(ip)) iok = true;
      }
      if (iok) {
        int iref = 1, itype = 0;
        if (use_quadtree) {
          iref = uv_flags_iref(ip);
          itype = uv_flags_type(ip);
        }
        int idir = uv_flags_dir(ip);
        T dxuvinv, dyuvinv, dxuv2inv, dyuv2inv;
        if (crsgeo) {  // sfincs_momentum.f90:205-234
          if (itype == 0) {
            if (idir == 0) {
              dxuvinv = dxminv(ip); dyuvinv = dyrinv(iref); dxuv2inv = dxm2inv(ip); dyuv2inv = dyr2inv(iref);
            } else {
              dxuvinv = dyrinv(iref); dyuvinv = dxminv(ip); dxuv2inv = dyr2inv(iref); dyuv2inv = dxm2inv(ip);
            }
          } else {
            if (idir == 0) {
              dxuvinv = (T)(1.0f / (3.0f * (1.0f / dxminv(ip)) / 2.0f)); dyuvinv = dyrinv(iref); dxuv2inv = 0;
              dyuv2inv = dyr2inv(iref);
            } else {
              dxuvinv = (T)(1.0f / (3.0f * (1.0f / dyrinv(iref)) / 2.0f)); dyuvinv = dxminv(ip); dxuv2inv = 0;
              dyuv2inv = dxm2inv(ip);
            }
          }
        } else if (itype == 0) {
          if (idir == 0) {
            dxuvinv = dxrinv(iref); dyuvinv = dyrinv(iref); dxuv2inv = dxr2inv(iref); dyuv2inv = dyr2inv(iref);
          } else {
            dxuvinv = dyrinv(iref); dyuvinv = dxrinv(iref); dxuv2inv = dyr2inv(iref); dyuv2inv = dxr2inv(iref);
          }
        } else {
          if (idir == 0) {
            dxuvinv = dxrinvc(iref); dyuvinv = dyrinv(iref); dxuv2inv = 0; dyuv2inv = dyr2inv(iref);
          } else {
            dxuvinv = dyrinvc(iref); dyuvinv = dxrinv(iref); dxuv2inv = 0; dyuv2inv = dxr2inv(iref);
          }
        }
        T fcoriouv = crsgeo ? (T)fcorio2d(nm) : (T)fcorio;
        T qx_nm = q0(ip);
        T qx_nmd = 0, qx_nmu = 0, qy_nm = 0, qy_nmu = 0, qy_ndm = 0, qy_ndmu = 0;
        T uu_nm = 0, uu_nmd = 0, uu_nmu = 0, uu_ndm = 0, uu_num = 0, vu = 0;
        if (advection || coriolis || viscosity || friction2d || thetasmoothing) {
          qx_nmd = q0(uv_index_u_nmd(ip));
          qx_nmu = q0(uv_index_u_nmu(ip));
          qy_nm = q0(uv_index_v_nm(ip));
          qy_nmu = q0(uv_index_v_nmu(ip));
          qy_ndm = q0(uv_index_v_ndm(ip));
          qy_ndmu = q0(uv_index_v_ndmu(ip));
          uu_nm = uv0(ip);
          uu_nmd = uv0(uv_index_u_nmd(ip));
          uu_nmu = uv0(uv_index_u_nmu(ip));
          uu_ndm = uv0(uv_index_u_ndm(ip));
          uu_num = uv0(uv_index_u_num(ip));
          vu = (uv0(uv_index_v_ndm(ip)) + uv0(uv_index_v_ndmu(ip)) + uv0(uv_index_v_nm(ip)) + uv0(uv_index_v_nmu(ip))) /
               (T)4;
        }
        T phi = 1;
        T hu, gnavg2;
        if (subgrid) {
          if (zsu > zmax && CORE) {
            hu = sg_uv_havg_zmax(ip) + zsu;
            gnavg2 = sg_uv_navg_w(ip) -
                     (sg_uv_navg_w(ip) - sg_uv_nrep_zmax(ip)) / std::fma(sg_uv_fnfit(ip), zsu - zmax, (T)1);
          } else if (zsu > zmax) {
            hu = sg_uv_havg_zmax(ip) + zsu;
            gnavg2 = sg_uv_navg_w(ip) -
                     (sg_uv_navg_w(ip) - sg_uv_nrep_zmax(ip)) / (sg_uv_fnfit(ip) * (zsu - zmax) + (T)1);
          } else if (CORE) {
            // scaled level x = (zsu - zmin) (L - 1) / (zmax - zmin): interval int(x) + 1, weight x - (iuv - 1)
            T rdz = (T)(L - 1) / (zmax - zmin);
            T x = (zsu - zmin) * rdz;
            long iuv = std::min(std::max((long)x + 1, 1L), L - 1);
            T facint = x - (T)(iuv - 1);
            hu = std::fma(sg_uv_havg(iuv + 1, ip) - sg_uv_havg(iuv, ip), facint, sg_uv_havg(iuv, ip));
            gnavg2 = std::fma(sg_uv_nrep(iuv + 1, ip) - sg_uv_nrep(iuv, ip), facint, sg_uv_nrep(iuv, ip));
            phi = std::fma(sg_uv_pwet(iuv + 1, ip) - sg_uv_pwet(iuv, ip), facint, sg_uv_pwet(iuv, ip));
          } else {
            T dzuv = (zmax - zmin) / (T)(L - 1);
            long iuv = std::min((long)((zsu - zmin) / dzuv) + 1, L - 1);
            T facint = (zsu - (zmin + (T)(iuv - 1) * dzuv)) / dzuv;
            hu = sg_uv_havg(iuv, ip) + (sg_uv_havg(iuv + 1, ip) - sg_uv_havg(iuv, ip)) * facint;
            gnavg2 = sg_uv_nrep(iuv, ip) + (sg_uv_nrep(iuv + 1, ip) - sg_uv_nrep(iuv, ip)) * facint;
            phi = sg_uv_pwet(iuv, ip) + (sg_uv_pwet(iuv + 1, ip) - sg_uv_pwet(iuv, ip)) * facint;
          }
        } else {
          hu = std::max(zsu - (T)zbuvmx(ip), (T)huthresh);
          gnavg2 = gn2uv(ip);
        }
        T hwet = hu / phi;
        T dzdx;
        if (slopelim < 9999.0f)
          dzdx = (T)std::min(std::max((T)((zs(nmu) - zs(nm)) * dxuvinv), (T)-slopelim), (T)slopelim);
        else
          dzdx = (T)((zs(nmu) - zs(nm)) * dxuvinv);
        T frc = -(T)g * hu * dzdx;
        if (advection) {
          if (mask_adv(ip) == 1) {
            T dqxudx = 0, dqyudy = 0;
            if (advection_scheme == 0) {
              if (qx_nm > (T)1.0e-6f)
                dqxudx = (qx_nm * uu_nm - qx_nmd * uu_nmd) * dxuvinv;
              else if (qx_nm < (T)-1.0e-6f)
                dqxudx = (qx_nmu * uu_nmu - qx_nm * uu_nm) * dxuvinv;
              T qy = qy_ndm + qy_ndmu + qy_nm + qy_nmu;
              if (qy > (T)1.0e-6f)
                dqyudy = (qy_ndm + qy_ndmu) * (uu_nm - uu_ndm) * dyuvinv / (T)2;
              else if (qy < (T)-1.0e-6f)
                dqyudy = (qy_nm + qy_nmu) * (uu_num - uu_nm) * dyuvinv / (T)2;
            } else {
              T qd = (qx_nmd + qx_nm) / (T)2;
              T qu = (qx_nm + qx_nmu) / (T)2;
              if (qd > (T)1.0e-6f) {
                T ud = (uu_nmd + uu_nm) / (T)2;
                dqxudx = (qd * (uu_nm - uu_nmd) + ud * (qx_nm - qx_nmd)) * dxuvinv;
              }
              if (qu < (T)-1.0e-6f) {
                T uu = (uu_nm + uu_nmu) / (T)2;
                dqxudx = dqxudx + (qu * (uu_nmu - uu_nm) + uu * (qx_nmu - qx_nm)) * dxuvinv;
              }
              qu = (qy_nm + qy_nmu) / (T)2;
              qd = (qy_ndm + qy_ndmu) / (T)2;
              if (qd > (T)1.0e-6f) dqyudy = qd * (uu_nm - uu_ndm) * dyuvinv;
              if (qu < (T)-1.0e-6f) dqyudy = dqyudy + qu * (uu_num - uu_nm) * dyuvinv;
              T ud = (uu_nmd + uu_nm) / (T)2;
              T uu = (uu_nm + uu_nmu) / (T)2;
              if (ud > (T)1.0e-6f) dqyudy = dqyudy + ud * (qy_nm - qy_ndm) * dyuvinv;
              if (uu < (T)-1.0e-6f) dqyudy = dqyudy + uu * (qy_nmu - qy_ndmu) * dyuvinv;
            }
            T adv = -phi * (dqxudx + dqyudy);
            adv = std::min(std::max(adv, -(T)advlim * hu), (T)advlim * hu);
            frc = frc + adv;
          }
        }
        if (viscosity) {
          T lap = (uu_nmu - (T)2 * uu_nm + uu_nmd) * dxuv2inv + (uu_num - (T)2 * uu_nm + uu_ndm) * dyuv2inv;
          if (itype == 0)
            frc = frc + (T)nuvisc(iref) * hu * lap;
          else
            frc = frc + (T)nuviscfac * (T)nuvisc(iref) * hu * lap;
        }
        if (coriolis) {
          if (idir == 0)
            frc = frc + fcoriouv * hu * vu;
          else
            frc = frc - fcoriouv * hu * vu;
        }
        if (wind) {
          T tw = idir == 0 ? (T)tauwu(nm) : (T)tauwv(nm);
          if (hwet > (T)0.25f)
            frc = frc + phi * tw;
          else
            frc = frc + tw * hu * (T)4;
        }
        if (patmos)  // atmospheric pressure gradient (sfincs_momentum.f90:585-589)
          frc = frc + hu * ((T)patm(nm) - (T)patm(nmu)) * dxuvinv / (T)rhow;
        T qfr;
        const T cr = CORE ? (T)core_cube_root((float)hu) : (T)0;  // the core's hu**(1/3)
        if (kfuv(ip) == 0) {
          T h53 = CORE ? hu * (cr * cr) : (T)std::pow(hu, (T)(5.0f / 3.0f));
          qfr = std::sqrt(std::fabs(dzdx) / (std::max(gnavg2, (T)1.0e-5f) / (T)10)) * h53;
        } else {
          if (friction2d && CORE) {
            T huvu = hu * vu;
            qfr = std::sqrt(std::fma(qx_nm, qx_nm, huvu * huvu));
          } else if (friction2d) {
            qfr = std::sqrt(qx_nm * qx_nm + (hu * vu) * (hu * vu));
          } else {
            qfr = std::fabs(qx_nm);
          }
        }
        T qsm = qx_nm;
        if (thetasmoothing) {
          if (kcuv(uv_index_u_nmd(ip)) == 1 && kcuv(uv_index_u_nmu(ip)) == 1) {
            if (std::fabs(qx_nmd) > (T)1.0e-6f && std::fabs(qx_nmu) > (T)1.0e-6f)
              qsm = (T)theta * qx_nm + (T)0.5f * ((T)1 - (T)theta) * (qx_nmu + qx_nmd);
          }
        }
        // The CUDA core evaluates hu**(1.0/3.0) as a cube root (under one ulp from
        // hu**0.333333343 for 1e-3 <= hu <= 1e3) and multiplies the flux update
        // through by hu73 (one division); the "f32" (core precision)
        // instantiation does the same, "ref" and "fp64" keep the reference's form.
        T hu73, qn;
        if (h73table) {
          hu73 = power7over3(std::max(hu, (T)1.0e-6f));
          qn = CORE ? (std::fma(frc, (T)dtt, qsm) * hu73) / std::fma(gnavg2 * (T)dtt, qfr, hu73)
                    : (qsm + frc * (T)dtt) / ((T)1 + gnavg2 * (T)dtt * qfr / hu73);
        } else if (CORE) {
          hu73 = (hu * hu) * cr;
          qn = (std::fma(frc, (T)dtt, qsm) * hu73) / std::fma(gnavg2 * (T)dtt, qfr, hu73);
        } else {
          hu73 = hu * hu * std::pow(hu, expo);
          qn = (qsm + frc * (T)dtt) / ((T)1 + gnavg2 * (T)dtt * qfr / hu73);
        }
        if (subgrid && wiggle_suppression) {
          T mdrv = std::fabs(zsderv(nm) - zsderv(nmu)) - (T)wiggle_threshold;
          if (mdrv > (T)0) qn = qn * (T)wiggle_threshold / ((T)wiggle_factor * mdrv + (T)wiggle_threshold);
        }
        if (subgrid) {
          if (z_volume(nm) < 0.0) qn = std::min(qn, (T)0);
          if (z_volume(nmu) < 0.0) qn = std::max(qn, (T)0);
        } else {
          if ((double)zs(nm) < (double)zb(nm)) qn = std::min(qn, (T)0);
          if ((double)zs(nmu) < (double)zb(nmu)) qn = std::max(qn, (T)0);
        }
        qn = std::min(std::max(qn, -hu * (T)uvlim), hu * (T)uvlim);
        q(ip) = qn;
        uv(ip) = qn / std::max(hu, (T)huvmin);
        kfuv(ip) = 1;
        T min_dt_ip = (T)1 / (std::max(std::sqrt((T)g * hu), std::fabs(uv(ip))) * dxuvinv);
        mdt = std::min(mdt, (float)min_dt_ip);
      } else {
        q(ip) = (T)0;
        uv(ip) = (T)0;
        kfuv(ip) = 0;
      }
    }
    min_dt = mdt;
    for (long ic = 1; ic <= ncuv; ic++) {
      q(cuv_index_uv(ic)) = (q(cuv_index_uv1(ic)) + q(cuv_index_uv2(ic))) / (T)2;
      uv(cuv_index_uv(ic)) = (uv(cuv_index_uv1(ic)) + uv(cuv_index_uv2(ic))) / (T)2;
    }
  }

  // compute_water_levels_regular: sfincs_continuity.f90:46-262
  void compute_water_levels_regular(float dtt, double tt) {
    for (long is = 1; is <= nsrcdrn; is++) {
      long nm = nmindsrc(is);
      zs(nm) = (TZ)std::max((double)(zs(nm) + (TZ)(qtsrc(is) * dtt / area_of(nm))), (double)zb(nm));
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (long nm = 1; nm <= np; nm++) {
      if (kcs(nm) == 1) {
        if (precip) zs(nm) = zs(nm) + (TZ)((T)netprcp(nm) * (T)dtt);
        if (use_qext) zs(nm) = zs(nm) + (TZ)((T)qext(nm) * (T)dtt);
        long nmd = z_index_uv_md(nm), nmu = z_index_uv_mu(nm), ndm = z_index_uv_nd(nm), num = z_index_uv_nu(nm);
        int ir = z_flags_iref(nm);
        T dz = crsgeo ? ((q(nmd) - q(nmu)) / (T)dxm(nm) + (q(ndm) - q(num)) * (T)dyrinv(ir)) * (T)dtt  // :135-147
                      : ((q(nmd) - q(nmu)) * (T)dxrinv(ir) + (q(ndm) - q(num)) * (T)dyrinv(ir)) * (T)dtt;
        zs(nm) = zs(nm) + (TZ)dz;
      }
      if (store_maximum_waterlevel) {
        if (store_t_zsmax && zs(nm) > zsmax(nm) && (zs(nm) - zb(nm)) > huthresh) t_zsmax(nm) = (float)tt;
        zsmax(nm) = (T)std::max((double)zsmax(nm), (double)zs(nm));
      }
    }
  }

  // compute_water_levels_subgrid: sfincs_continuity.f90:265-624
  void compute_water_levels_subgrid(float dtt, double tt) {
    for (long is = 1; is <= nsrcdrn; is++) {
      long nm = nmindsrc(is);
      if (z_volume(nm) >= 0.0 || (qtsrc(is) < 0.0f && z_volume(nm) >= 0.0))
        z_volume(nm) = z_volume(nm) + (TV)(qtsrc(is) * dtt);
    }
    const long L = subgrid_nlevels;
#pragma omp parallel for schedule(dynamic, 256)
    for (long nm = 1; nm <= np; nm++) {
      T dvol = 0;
      if (kcs(nm) == 1) {
        long nmd = z_index_uv_md(nm), nmu = z_index_uv_mu(nm), ndm = z_index_uv_nd(nm), num = z_index_uv_nu(nm);
        if (crsgeo) {  // :350-361
          int ir = z_flags_iref(nm);
          dvol = dvol + ((q(nmd) - q(nmu)) * (T)dyrm(ir) + (q(ndm) - q(num)) * (T)dxm(nm)) * (T)dtt;
        } else if (use_quadtree) {
          int ir = z_flags_iref(nm);
          dvol = dvol + ((q(nmd) - q(nmu)) * (T)dyrm(ir) + (q(ndm) - q(num)) * (T)dxrm(ir)) * (T)dtt;
        } else {
          dvol = dvol + ((q(nmd) - q(nmu)) * (T)dy + (q(ndm) - q(num)) * (T)dx) * (T)dtt;
        }
      }
      if (kcs(nm) == 1 || kcs(nm) == 4) {
        T a = area_of(nm);  // :458-470
        if (precip || use_qext) {
          T dzsdt = 0;
          if (precip) dzsdt = dzsdt + (T)netprcp(nm);
          if (use_qext) dzsdt = dzsdt + (T)qext(nm);
          dvol = dvol + dzsdt * a * (T)dtt;
        }
        z_volume(nm) = z_volume(nm) + (TV)dvol;
        T zs00 = 0, zs11 = 0;
        if (wiggle_suppression) {
          zs00 = zs0(nm);
          zs11 = (T)zs(nm);
          zs0(nm) = zs11;
        }
        if (z_volume(nm) >= (TV)(sg_z_volmax(nm) * 0.999f)) {
          zs(nm) = (TZ)((TV)std::max(sg_z_zmax(nm), -20.0f) + (z_volume(nm) - (TV)sg_z_volmax(nm)) / (TV)a);
        } else if (z_volume(nm) <= (TV)1.0e-6f) {
          zs(nm) = (TZ)std::max(sg_z_zmin(nm), -20.0f);
        } else {
          T dzvol = (T)sg_z_volmax(nm) / (T)(L - 1);
          long iuv = (long)(z_volume(nm) / (TV)dzvol) + 1;
          T facint = (T)((z_volume(nm) - (TV)((T)(iuv - 1) * dzvol)) / (TV)dzvol);
          zs(nm) = (TZ)((T)sg_z_dep(iuv, nm) + ((T)sg_z_dep(iuv + 1, nm) - (T)sg_z_dep(iuv, nm)) * facint);
        }
        // zs is real*8 in the reference: zs - 2*zs11 + zs00 is evaluated in TZ precision
        if (wiggle_suppression) zsderv(nm) = (T)(zs(nm) - (TZ)((T)2 * zs11) + (TZ)zs00);
      }
      if (store_maximum_waterlevel) {
        if (store_t_zsmax && zs(nm) > zsmax(nm) && (zs(nm) - sg_z_zmin(nm)) > huthresh) t_zsmax(nm) = (float)tt;
        zsmax(nm) = (T)std::max((double)zsmax(nm), (double)zs(nm));
      }
    }
  }

  // compute_store_variables: sfincs_continuity.f90:626-720
  void compute_store_variables(float dtt) {
    for (long nm = 1; nm <= np; nm++) {
      T qz = 0, uvz = 0;
      if (kcs(nm) == 1 || kcs(nm) == 4) {
        long nmd = z_index_uv_md(nm), nmu = z_index_uv_mu(nm), ndm = z_index_uv_nd(nm), num = z_index_uv_nu(nm);
        if (store_maximum_velocity) {
          T quz = (uv(nmd) + uv(nmu)) / (T)2, qvz = (uv(ndm) + uv(num)) / (T)2;
          uvz = std::sqrt(quz * quz + qvz * qvz);
          vmax(nm) = std::max(vmax(nm), uvz);
        }
        if (store_maximum_flux) {
          T quz = (q(nmd) + q(nmu)) / (T)2, qvz = (q(ndm) + q(num)) / (T)2;
          qz = std::sqrt(quz * quz + qvz * qvz);
          qmax(nm) = std::max(qmax(nm), qz);
        }
        if (store_twet) {
          double base = subgrid ? (double)sg_z_zmin(nm) : (double)zb(nm);
          if ((double)zs(nm) - base > (double)twet_threshold) twet(nm) = twet(nm) + (T)dtt;
        }
      }
    }
  }

  // sfincs_update: sfincs_lib.f90:337-683 (output and optional processes elided)
  int update(double dtrange, long max_steps = -1) {
    double tend;
    bool single = false;
    if (dtrange < -999.0)
      tend = t1;
    else if (dtrange <= 0.0) {
      tend = t1;
      single = true;
    } else
      tend = t + dtrange;
    long done = 0;
    while (t < tend) {
      if (max_steps >= 0 && done >= max_steps) break;
      nt++;
      dt = alfa * min_dt;
      float dtchk = alfa * min_dt;
      t = t + (double)dt;
      dtavg = dtavg + dt;
      bool write_max = false;  // sfincs_lib.f90:430-445
      if (t >= tmaxout) {
        write_max = true;
        ntmaxout++;
        if (t < (double)t1) tmaxout = tmaxout + (double)dtmaxout;
      }
      bool update_meteo = false;  // sfincs_lib.f90:493-503
      if (meteo3d && t >= (double)twindupd) {
        meteo_t0 = twindupd;
        meteo_t1 = twindupd + dtwindupd;
        twindupd = twindupd + dtwindupd;
        update_meteo = true;
      }
      if (wind || patmos || precip) {
        if (meteo3d && update_meteo) update_meteo_fields();
        update_meteo_forcing(t, dt);
        if (infiltration) update_infiltration_map(dt);
      }
      if (boundaries_in_mask) {
        if (nbnd > 0) update_boundary_points(t);
        update_boundary_conditions(t);
        update_boundary_fluxes(dt, t);
      }
      update_discharges(t);
      compute_fluxes(dt);
      if (nrstructures > 0) compute_fluxes_over_structures();
      if (subgrid)
        compute_water_levels_subgrid(dt, t);
      else
        compute_water_levels_regular(dt, t);
      if (store_maximum_velocity || store_maximum_flux || store_twet) compute_store_variables(dt);
      if (write_max) {  // write_output: the max fields as written, then reset (sfincs_output.f90:158-230)
        if (store_maximum_waterlevel) {
          zsmax_out = zsmax;
          zsmax.fill((T)-999.0f);
        }
        if (store_maximum_velocity) {
          vmax_out = vmax;
          vmax.fill((T)-999.0f);
        }
        if (store_maximum_flux) {
          qmax_out = qmax;
          qmax.fill((T)-999.0f);
        }
        if (store_twet) {
          twet_out = twet;
          twet.fill((T)0.0f);
        }
        if (store_t_zsmax) {
          tzsmax_out = t_zsmax;
          t_zsmax.fill(-999.0f);
        }
      }
      if (dtchk < dtmin && nt > 1) {
        error = 1;
        t = (double)t1 + 1.0;
      }
      done++;
      if (single) tend = t0;
    }
    return 0;
  }
};

struct Handle {
  std::string precision;
  void* m = nullptr;
  std::string err;
};

}  // namespace orc

using namespace orc;
using M64 = Model<double, double, double>;
using MRef = Model<float, double, double>;
using M32 = Model<float, float, double>;

template <class Fn>
static auto dispatch(Handle* h, Fn fn) {
  if (h->precision == "fp64") return fn(*static_cast<M64*>(h->m));
  if (h->precision == "ref") return fn(*static_cast<MRef*>(h->m));
  return fn(*static_cast<M32*>(h->m));
}

template <class A, class X>
static void copy_out(const F1<A>& a, X* out, long n) {
  for (long i = 0; i < n; i++) out[i] = (X)a((long)i + 1);
}

static thread_local std::string g_last_error;

extern "C" {

// Create and initialise a model from <dir>/sfincs.inp.  precision: "fp64", "ref", "f32".
// bmi != 0 mirrors the BMI initialize() (use_qext on).  Returns NULL on error.
void* oracle_create(const char* dir, const char* precision, int bmi) {
  auto* h = new Handle();
  h->precision = precision;
  try {
    if (h->precision == "fp64") {
      auto* m = new M64();
      h->m = m;
      m->initialize(dir, bmi != 0);
    } else if (h->precision == "ref") {
      auto* m = new MRef();
      h->m = m;
      m->initialize(dir, bmi != 0);
    } else if (h->precision == "f32") {
      auto* m = new M32();
      h->m = m;
      m->initialize(dir, bmi != 0);
    } else {
      throw std::runtime_error("unknown precision");
    }
  } catch (std::exception& e) {
    g_last_error = e.what();
    return nullptr;
  }
  return h;
}

const char* oracle_last_error() { return g_last_error.c_str(); }

// The core's arctangent (IEEE operations only), for its accuracy test.
float oracle_core_atan2(float y, float x) { return core_atan2(y, x); }
double oracle_core_cos(double x) { return core_cos(x); }

void oracle_destroy(void* hv) {
  auto* h = static_cast<Handle*>(hv);
  if (!h) return;
  dispatch(h, [&](auto& m) {
    delete &m;
    return 0;
  });
  delete h;
}

// sfincs_update(dtrange) semantics; max_steps < 0 means unbounded.  Returns steps taken.
long oracle_update(void* hv, double dtrange, long max_steps) {
  auto* h = static_cast<Handle*>(hv);
  return dispatch(h, [&](auto& m) {
    long n0 = m.nt;
    m.update(dtrange, max_steps);
    return m.nt - n0;
  });
}

// Scalars: [t, dt, min_dt, t0, t1, nt, error, dtmax, dtmin, np, npuv, nkcuv2, ngbnd, subgrid, nlevels]
void oracle_scalars(void* hv, double* out) {
  auto* h = static_cast<Handle*>(hv);
  dispatch(h, [&](auto& m) {
    double v[] = {m.t, m.dt, m.min_dt, m.t0, m.t1, (double)m.nt, (double)m.error, m.dtmax, m.dtmin,
                  (double)m.np, (double)m.npuv, (double)m.nkcuv2, (double)m.ngbnd, (double)m.subgrid,
                  (double)m.subgrid_nlevels};
    std::memcpy(out, v, sizeof(v));
    return 0;
  });
}

// Copy a named array to a double buffer of length n (cells: np, faces: npuv).
// Names: zs zsmax vmax qmax twet tzsmax z_volume zs0 zsderv zb z_zmin kcs nm_n nm_m q uv kfuv kcuv uv_nm uv_nmu uv_dir netprcp qext
int oracle_get(void* hv, const char* name, double* out, long n) {
  auto* h = static_cast<Handle*>(hv);
  std::string s(name);
  return dispatch(h, [&](auto& m) -> int {
    if (s == "zs") copy_out(m.zs, out, n);
    else if (s == "zsmax" && m.zsmax.allocated()) copy_out(m.zsmax, out, n);
    else if (s == "vmax" && m.vmax.allocated()) copy_out(m.vmax, out, n);
    else if (s == "qmax" && m.qmax.allocated()) copy_out(m.qmax, out, n);
    else if (s == "twet" && m.twet.allocated()) copy_out(m.twet, out, n);
    else if (s == "tzsmax" && m.t_zsmax.allocated()) copy_out(m.t_zsmax, out, n);
    else if (s == "z_volume" && m.z_volume.allocated()) copy_out(m.z_volume, out, n);
    else if (s == "zs0" && m.zs0.allocated()) copy_out(m.zs0, out, n);
    else if (s == "zsderv" && m.zsderv.allocated()) copy_out(m.zsderv, out, n);
    else if (s == "zb" && m.zb.allocated()) copy_out(m.zb, out, n);
    else if (s == "z_zmin" && m.sg_z_zmin.allocated()) copy_out(m.sg_z_zmin, out, n);
    else if (s == "kcs") copy_out(m.kcs, out, n);
    else if (s == "nm_n") copy_out(m.z_index_z_n, out, n);
    else if (s == "nm_m") copy_out(m.z_index_z_m, out, n);
    else if (s == "q") copy_out(m.q, out, n);
    else if (s == "uv") copy_out(m.uv, out, n);
    else if (s == "kfuv") copy_out(m.kfuv, out, n);
    else if (s == "kcuv") copy_out(m.kcuv, out, n);
    else if (s == "mask_adv" && m.mask_adv.allocated()) copy_out(m.mask_adv, out, n);
    else if (s == "uv_nm") copy_out(m.uv_index_z_nm, out, n);
    else if (s == "uv_nmu") copy_out(m.uv_index_z_nmu, out, n);
    else if (s == "uv_dir") copy_out(m.uv_flags_dir, out, n);
    else if (s == "uv_iref" && m.uv_flags_iref.allocated()) copy_out(m.uv_flags_iref, out, n);
    else if (s == "uv_type" && m.uv_flags_type.allocated()) copy_out(m.uv_flags_type, out, n);
    else if (s == "uv_u_nmd" && m.uv_index_u_nmd.allocated()) copy_out(m.uv_index_u_nmd, out, n);
    else if (s == "uv_u_nmu" && m.uv_index_u_nmu.allocated()) copy_out(m.uv_index_u_nmu, out, n);
    else if (s == "uv_u_ndm" && m.uv_index_u_ndm.allocated()) copy_out(m.uv_index_u_ndm, out, n);
    else if (s == "uv_u_num" && m.uv_index_u_num.allocated()) copy_out(m.uv_index_u_num, out, n);
    else if (s == "uv_v_ndm" && m.uv_index_v_ndm.allocated()) copy_out(m.uv_index_v_ndm, out, n);
    else if (s == "uv_v_nm" && m.uv_index_v_nm.allocated()) copy_out(m.uv_index_v_nm, out, n);
    else if (s == "uv_v_ndmu" && m.uv_index_v_ndmu.allocated()) copy_out(m.uv_index_v_ndmu, out, n);
    else if (s == "uv_v_nmu" && m.uv_index_v_nmu.allocated()) copy_out(m.uv_index_v_nmu, out, n);
    else if (s == "z_uv_md") copy_out(m.z_index_uv_md, out, n);
    else if (s == "z_uv_mu") copy_out(m.z_index_uv_mu, out, n);
    else if (s == "z_uv_nd") copy_out(m.z_index_uv_nd, out, n);
    else if (s == "z_uv_nu") copy_out(m.z_index_uv_nu, out, n);
    else if (s == "cuv_uv1" && m.ncuv > 0) copy_out(m.cuv_index_uv1, out, n);
    else if (s == "cuv_uv2" && m.ncuv > 0) copy_out(m.cuv_index_uv2, out, n);
    else if (s == "zbuvmx" && m.zbuvmx.allocated()) copy_out(m.zbuvmx, out, n);
    else if (s == "gn2uv" && m.gn2uv.allocated()) copy_out(m.gn2uv, out, n);
    else if (s == "netprcp" && m.netprcp.allocated()) copy_out(m.netprcp, out, n);
    else if (s == "prcp" && m.prcp.allocated()) copy_out(m.prcp, out, n);
    else if (s == "cumprcp" && m.cumprcp.allocated()) copy_out(m.cumprcp, out, n);
    else if (s == "cuminf" && m.cuminf.allocated()) copy_out(m.cuminf, out, n);
    else if (s == "qext" && m.qext.allocated()) copy_out(m.qext, out, n);
    else if (s == "uvmean") copy_out(m.uvmean, out, n);
    else if (s == "cell_area_m2" && m.cell_area_m2.allocated()) copy_out(m.cell_area_m2, out, n);
    else if (s == "dxm" && m.dxm.allocated()) copy_out(m.dxm, out, n);
    else if (s == "zsmax_out" && m.zsmax_out.allocated()) copy_out(m.zsmax_out, out, n);
    else if (s == "vmax_out" && m.vmax_out.allocated()) copy_out(m.vmax_out, out, n);
    else if (s == "qmax_out" && m.qmax_out.allocated()) copy_out(m.qmax_out, out, n);
    else if (s == "twet_out" && m.twet_out.allocated()) copy_out(m.twet_out, out, n);
    else if (s == "tzsmax_out" && m.tzsmax_out.allocated()) copy_out(m.tzsmax_out, out, n);
    else if (s == "ntmaxout") out[0] = (double)m.ntmaxout;
    else if (s == "tauwu0" && m.tauwu0.allocated()) copy_out(m.tauwu0, out, n);
    else if (s == "tauwv0" && m.tauwv0.allocated()) copy_out(m.tauwv0, out, n);
    else if (s == "tauwu1" && m.tauwu1.allocated()) copy_out(m.tauwu1, out, n);
    else if (s == "tauwv1" && m.tauwv1.allocated()) copy_out(m.tauwv1, out, n);
    else if (s == "patm0" && m.patm0.allocated()) copy_out(m.patm0, out, n);
    else if (s == "patm1" && m.patm1.allocated()) copy_out(m.patm1, out, n);
    else if (s == "prcp0" && m.prcp0.allocated()) copy_out(m.prcp0, out, n);
    else if (s == "prcp1" && m.prcp1.allocated()) copy_out(m.prcp1, out, n);
    else if (s == "nrstructures") out[0] = (double)m.nrstructures;
    else if (s == "struc") {
      // per structure: uv point (1-based), crest level, Cd, relative length
      for (long i = 1; i <= m.nrstructures && 4 * (i - 1) + 3 < n; i++) {
        out[4 * (i - 1)] = m.structure_uv_index(i);
        out[4 * (i - 1) + 1] = m.structure_parameters(1, i);
        out[4 * (i - 1) + 2] = m.structure_parameters(2, i);
        out[4 * (i - 1) + 3] = m.structure_length(i);
      }
    }
    else if (s == "crs_faces") {  // per crossed uv point: cross-section, cell nm (0-based), direction, sign
      long k = 0;
      for (size_t c = 0; c < m.crs_uv_index.size(); c++)
        for (size_t j = 0; j < m.crs_uv_index[c].size(); j++) {
          if (4 * k + 3 >= n) return -1;
          const long ip = m.crs_uv_index[c][j];
          out[4 * k] = (double)c;
          out[4 * k + 1] = (double)(m.uv_index_z_nm(ip) - 1);
          out[4 * k + 2] = (double)m.uv_flags_dir(ip);
          out[4 * k + 3] = (double)m.crs_idir[c][j];
          k++;
        }
      if (4 * k != n) return -1;
    }
    else if (s == "q_drain") {  // per drainage structure the rate of its intake entry (sfincs_ncoutput.F90:1410-1421)
      if (m.ndrn != n) return -1;
      for (long i = 1; i <= n; i++) out[i - 1] = (double)m.qtsrc(m.nsrc + 2 * i - 1);
    }
    else if (s == "runup_zs") {  // run-up level of every gauge from the current zs
      if ((long)m.runup_gauge_nm.size() != n) return -1;
      for (long i = 0; i < n; i++) out[i] = (double)m.runup_level((size_t)i);
    }
    else if (s == "crs_discharge") {  // discharge through every cross-section from the current q
      if ((long)m.namecrs.size() != n) return -1;
      for (long i = 0; i < n; i++) out[i] = (double)m.crs_discharge((size_t)i);
    }
    else if (s == "tide_omega" || s == "tide_amp" || s == "tide_phase") {
      // astronomic constituents after the nodal correction: per constituent, or per point and constituent
      const std::vector<double>& src =
          s == "tide_omega" ? m.tidal_component_frequency : (s == "tide_amp" ? m.tidal_amp : m.tidal_phase);
      if ((long)src.size() != n) return -1;
      for (long i = 0; i < n; i++) out[i] = src[(size_t)i];
    }
    else if (s == "kb_cell" || s == "kb_dir" || s == "kb_sign") {
      // water-level boundary faces (kcuv==2/6 list without lateral Neumann faces), reference order
      long k = 0;
      for (long ib = 1; ib <= m.nkcuv2; ib++) {
        if (m.kcs(m.nmbkcuv2(ib)) == 6) continue;
        if (k >= n) return -1;
        long ip = m.index_kcuv2(ib);
        if (s == "kb_cell") out[k] = (double)(m.uv_index_z_nm(ip) - 1);
        else if (s == "kb_dir") out[k] = (double)m.uv_flags_dir(ip);
        else out[k] = (double)m.ibuvdir(ib);
        k++;
      }
      if (k != n) return -1;
    }
    else return -1;
    return 0;
  });
}

// Overwrite a named state array from a double buffer (zs, q, uv, qext, zsmax, z_volume).
int oracle_set(void* hv, const char* name, const double* in, long n) {
  auto* h = static_cast<Handle*>(hv);
  std::string s(name);
  return dispatch(h, [&](auto& m) -> int {
    using MT = std::remove_reference_t<decltype(m)>;
    auto put = [&](auto& arr) {
      using X = std::remove_reference_t<decltype(arr(1))>;
      for (long i = 0; i < n; i++) arr((long)i + 1) = (X)in[i];
    };
    (void)sizeof(MT);
    if (s == "zs") put(m.zs);
    else if (s == "q") put(m.q);
    else if (s == "uv") put(m.uv);
    else if (s == "qext" && m.qext.allocated()) put(m.qext);
    else if (s == "z_volume" && m.z_volume.allocated()) put(m.z_volume);
    else return -1;
    return 0;
  });
}

}  // extern "C"
