// Flux update of one uv face (sfincs_momentum.f90:389-733), shared by the
// regular-grid tile kernels and the quadtree face kernels.
#pragma once
#include <cfloat>
#include <cstdint>

#include "sfg_device.h"

namespace sfg {

// Cube root of a float from IEEE additions, multiplications and fused
// multiply-adds only, so that the oracle reproduces it bit for bit on the CPU
// (std::fma is the same correctly rounded operation).  Method: an estimate of
// x^(-1/3) from the exponent (the float's bit pattern divided by three,
// reflected about a constant chosen here to minimise the estimate's worst
// relative error, 3.4 %), two Newton steps r += r (1 - x r^3) / 3 for
// x^(-1/3), y = x r^2, and one Newton correction of y.  At most 0.75 ulp from
// the exact cube root for 7.5e-9 <= x <= 32768, at most 1.1 ulp over all
// positive floats (denormals are scaled by 2^72 first); the reference's
// hu**(1.0/3.0) is a float power with its own rounding.  0, infinity and NaN
// pass through; negative x gives -cube_root(-x).
__device__ __forceinline__ float cube_root_pos(float x) {
  float s = 1.0f;
  if (x < 1.17549435e-38f) {  // below the smallest normal float
    x = x * 4722366482869645213696.0f;  // 2^72
    s = 5.9604644775390625e-08f;        // 2^-24
  }
  float r = __uint_as_float(0x54a232a0u - __float_as_uint(x) / 3u);
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const float r3 = (r * r) * r;
    const float e = fmaf(-x, r3, 1.0f);
    r = fmaf(r * 0.333333343f, e, r);
  }
  float y = (x * r) * r;
  const float res = fmaf(-(y * y), y, x);
  y = fmaf(res * 0.333333343f, r * r, y);
  return y * s;
}
__device__ __forceinline__ float cube_root(float x) {
  if (x > 0.0f && x < 3.40282347e+38f) return cube_root_pos(x);
  if (x < 0.0f && x > -3.40282347e+38f) return -cube_root_pos(-x);
  return x + x;  // 0, +-infinity, NaN
}

// Subgrid table interval and weight of a face level zsu (sfincs_momentum.f90:
// 370-378).  The reference divides three times by dzuv = (zmax - zmin) /
// (nlev - 1); here the scaled level x = (zsu - zmin) * ((nlev - 1) / (zmax -
// zmin)) takes one division, the interval is int(x) + 1 and the weight is
// x - (iuv - 1), the same quantity up to rounding.
struct SgLevel {
  int iuv;
  float facint;
};
__device__ __forceinline__ SgLevel sg_level(float zsu, float zmin, float zmax, int nlev) {
  const float rdz = (float)(nlev - 1) / (zmax - zmin);
  const float x = (zsu - zmin) * rdz;
  const int iuv = lev_index(x, nlev);
  return SgLevel{iuv, x - (float)(iuv - 1)};
}
// Roughness above the table (sfincs_momentum.f90:351-364).
__device__ __forceinline__ float sg_gnavg2_full(float navg, float nrep_zmax, float fnfit, float dz) {
  return navg - (navg - nrep_zmax) / fmaf(fnfit, dz, 1.0f);
}

// hu**(7/3) from the lookup table (power7over3, sfincs_momentum.f90:787-820):
// decade k of hu (1e-5 .. 1e4) picks column k, and int(10**(8 - k + 1) hu)
// the row.  The row is clamped to 1..1000; the reference reads outside its
// table if rounding lands a value just below a decade boundary on row 1000 +.
__device__ __forceinline__ float power7over3(float hu, const float* __restrict__ x73) {
  int k;
  float sc;
  if (hu < 0.00001f) { k = 1; sc = 1e8f; }
  else if (hu < 0.0001f) { k = 2; sc = 1e7f; }
  else if (hu < 0.001f) { k = 3; sc = 1e6f; }
  else if (hu < 0.01f) { k = 4; sc = 1e5f; }
  else if (hu < 0.1f) { k = 5; sc = 1e4f; }
  else if (hu < 1.0f) { k = 6; sc = 1e3f; }
  else if (hu < 10.0f) { k = 7; sc = 100.0f; }
  else if (hu < 100.0f) { k = 8; sc = 10.0f; }
  else if (hu < 1000.0f) { k = 9; sc = 1.0f; }
  else if (hu < 10000.0f) { k = 10; sc = 0.1f; }
  else return 2154433024.0f;  // 10000.0**(7.0/3.0) in real*4
  const int j = min(max((int)(sc * hu), 1), 1000);
  return __ldg(x73 + (k - 1) * 1000 + (j - 1));
}

// Wind stress and pressure difference of a face between storage cells c (nm)
// and cu (nmu) this step: the uniform wind of a time series unless the wind
// comes from a gridded field (then the value of cell nm), and patm(nm) -
// patm(nmu) from the gridded pressure.
__device__ __forceinline__ void face_meteo(const ScnDev& S, const StepVals& sv, int dir, int64_t c, int64_t cu,
                                           float& tauw, float& dpatm) {
  tauw = dir == 0 ? sv.twu : sv.twv;
  dpatm = 0.0f;
  if (S.wind_field | S.patmos) {
    const StepState& st = *S.st;
    const MeteoW w = meteo_weights(S, st.t, st.meteo_t0, st.meteo_t1);
    if (S.wind_field) tauw = cell_tau(S, c, dir, w);
    if (S.patmos) dpatm = cell_patm(S, c, w) - cell_patm(S, cu, w);
  }
}

// Grid spacing of one face (sfincs_momentum.f90:205-313): across the face
// (dxuv), along it (dyuv), their squared inverses for viscosity, and the
// viscosity coefficient of the face's refinement level.
struct FaceGeo {
  float dxuvinv, dyuvinv, dxuv2inv, dyuv2inv, nuvisc;
  float fcorio;  // Coriolis parameter at the face (per cell on geographic grids)
};

// Gathered inputs of one face (sfincs_momentum.f90:317-335 naming).
struct FaceV {
  float qx_nm, qx_nmd, qx_nmu, qy_nm, qy_nmu, qy_ndm, qy_ndmu;
  float uu_nm, uu_nmd, uu_nmu, uu_ndm, uu_num, vu;
};

// Flux update of one wet face from gathered inputs (sfincs_momentum.f90:389-733).
// Writes q, uv and returns g*hu.  The face's CFL denominator is
// den = max(sqrt(g*hu), |uv|) * dxuvinv and the reference takes the minimum of
// 1/den over faces (:731-733).  Correctly rounded division, square root and
// multiplication by a positive constant are monotone, so that minimum equals
// 1 / (max(sqrt(max g*hu), max |uv|) * dxuvinv) over faces of equal spacing,
// bit for bit: callers fold g*hu and |uv| and take one square root and one
// division per reduction instead of per face.
// tauw: the wind stress of the face's cell nm in the face direction (uniform
// from a time series, or the cell's value of the gridded field); dpatm:
// patm(nm) - patm(nmu) when atmospheric pressure is on.
template <bool SG>
__device__ __forceinline__ float face_flux_geo(const ScnDev& S, const StepVals& st, int dir, bool adv_on,
                                               bool theta_on, const FaceGeo& geo, uint8_t kf, float zs_nm,
                                               float zs_nmu, float hu, float gnavg2, float phi, const FaceV& a,
                                               bool dry_nm, bool dry_nmu, float zd_nm, float zd_nmu, float tauw,
                                               float dpatm, float& q_out, float& uv_out) {
  const float dxuvinv = geo.dxuvinv, dyuvinv = geo.dyuvinv, dxuv2inv = geo.dxuv2inv, dyuv2inv = geo.dyuv2inv;
  float dzdx;
  if (S.slopelim < 9999.0f)
    dzdx = fminf(fmaxf((zs_nmu - zs_nm) * dxuvinv, -S.slopelim), S.slopelim);
  else
    dzdx = (zs_nmu - zs_nm) * dxuvinv;
  float frc = -S.g * hu * dzdx;
  if (S.advection && adv_on) {
    float dqxudx = 0.0f, dqyudy = 0.0f;
    if (S.adv_scheme == 0) {
      if (a.qx_nm > 1.0e-6f)
        dqxudx = (a.qx_nm * a.uu_nm - a.qx_nmd * a.uu_nmd) * dxuvinv;
      else if (a.qx_nm < -1.0e-6f)
        dqxudx = (a.qx_nmu * a.uu_nmu - a.qx_nm * a.uu_nm) * dxuvinv;
      const float qy = a.qy_ndm + a.qy_ndmu + a.qy_nm + a.qy_nmu;
      if (qy > 1.0e-6f)
        dqyudy = (a.qy_ndm + a.qy_ndmu) * (a.uu_nm - a.uu_ndm) * dyuvinv / 2.0f;
      else if (qy < -1.0e-6f)
        dqyudy = (a.qy_nm + a.qy_nmu) * (a.uu_num - a.uu_nm) * dyuvinv / 2.0f;
    } else {
      float qd = (a.qx_nmd + a.qx_nm) / 2.0f;
      float qu = (a.qx_nm + a.qx_nmu) / 2.0f;
      if (qd > 1.0e-6f) {
        const float ud = (a.uu_nmd + a.uu_nm) / 2.0f;
        dqxudx = (qd * (a.uu_nm - a.uu_nmd) + ud * (a.qx_nm - a.qx_nmd)) * dxuvinv;
      }
      if (qu < -1.0e-6f) {
        const float uu = (a.uu_nm + a.uu_nmu) / 2.0f;
        dqxudx = dqxudx + (qu * (a.uu_nmu - a.uu_nm) + uu * (a.qx_nmu - a.qx_nm)) * dxuvinv;
      }
      qu = (a.qy_nm + a.qy_nmu) / 2.0f;
      qd = (a.qy_ndm + a.qy_ndmu) / 2.0f;
      if (qd > 1.0e-6f) dqyudy = qd * (a.uu_nm - a.uu_ndm) * dyuvinv;
      if (qu < -1.0e-6f) dqyudy = dqyudy + qu * (a.uu_num - a.uu_nm) * dyuvinv;
      const float ud = (a.uu_nmd + a.uu_nm) / 2.0f;
      const float uu = (a.uu_nm + a.uu_nmu) / 2.0f;
      if (ud > 1.0e-6f) dqyudy = dqyudy + ud * (a.qy_nm - a.qy_ndm) * dyuvinv;
      if (uu < -1.0e-6f) dqyudy = dqyudy + uu * (a.qy_nmu - a.qy_ndmu) * dyuvinv;
    }
    float adv = -phi * (dqxudx + dqyudy);
    adv = fminf(fmaxf(adv, -S.advlim * hu), S.advlim * hu);
    frc = frc + adv;
  }
  if (S.viscosity) {
    frc = frc + geo.nuvisc * hu *
                    ((a.uu_nmu - 2.0f * a.uu_nm + a.uu_nmd) * dxuv2inv +
                     (a.uu_num - 2.0f * a.uu_nm + a.uu_ndm) * dyuv2inv);
  }
  if (S.coriolis) {
    if (dir == 0)
      frc = frc + geo.fcorio * hu * a.vu;
    else
      frc = frc - geo.fcorio * hu * a.vu;
  }
  if (S.wind) {
    const float hwet = hu / phi;
    if (hwet > 0.25f)
      frc = frc + phi * tauw;
    else
      frc = frc + tauw * hu * 4.0f;
  }
  if (S.patmos) frc = frc + hu * dpatm * dxuvinv / S.rhow;  // atmospheric pressure (:585-589)
  // hu**(1.0/3.0) (:616, :673) as a cube root; the real*4 exponent 1.0/3.0 is
  // 0.333333343, so the two differ by a factor hu**(1e-8), under one ulp for
  // 1e-3 <= hu <= 1e3
  const float c = cube_root(hu);
  float qfr;
  if (!(kf & KF_WET)) {
    // hu**(5.0/3.0) = hu * (hu**(1/3))**2
    qfr = sqrtf(fabsf(dzdx) / (fmaxf(gnavg2, 1.0e-5f) / 10.0f)) * (hu * (c * c));
  } else if (S.friction2d) {
    const float huvu = hu * a.vu;
    qfr = sqrtf(fmaf(a.qx_nm, a.qx_nm, huvu * huvu));
  } else {
    qfr = fabsf(a.qx_nm);
  }
  float qsm = a.qx_nm;
  if (S.thetasmooth && theta_on && fabsf(a.qx_nmd) > 1.0e-6f && fabsf(a.qx_nmu) > 1.0e-6f)
    qsm = S.theta * a.qx_nm + 0.5f * (1.0f - S.theta) * (a.qx_nmu + a.qx_nmd);
  const float dt = st.dt;
  // q = (qsm + frc dt) / (1 + gnavg2 dt qfr / hu73) (:677), multiplied through
  // by hu73 = hu**2 * hu**(1/3) (:673) so that it takes one division
  const float hu73 = S.h73table ? power7over3(fmaxf(hu, 1.0e-6f), S.x73) : (hu * hu) * c;
  float q = (fmaf(frc, dt, qsm) * hu73) / fmaf(gnavg2 * dt, qfr, hu73);
  if (SG && S.wiggle) {
    const float mdrv = fabsf(zd_nm - zd_nmu) - S.wiggle_threshold;
    if (mdrv > 0.0f) q = q * S.wiggle_threshold / (S.wiggle_factor * mdrv + S.wiggle_threshold);
  }
  if (dry_nm) q = fminf(q, 0.0f);
  if (dry_nmu) q = fmaxf(q, 0.0f);
  q = fminf(fmaxf(q, -hu * S.uvlim), hu * S.uvlim);
  const float uv = q / fmaxf(hu, S.huvmin);
  q_out = q;
  uv_out = uv;
  return S.g * hu;
}

}  // namespace sfg
