// Flux update of one uv face (sfincs_momentum.f90:389-733), shared by the
// regular-grid tile kernels and the quadtree face kernels.
#pragma once
#include <cfloat>
#include <cstdint>

#include "sfg_device.h"

namespace sfg {

// Grid spacing of one face (sfincs_momentum.f90:205-313): across the face
// (dxuv), along it (dyuv), their squared inverses for viscosity, and the
// viscosity coefficient of the face's refinement level.
struct FaceGeo {
  float dxuvinv, dyuvinv, dxuv2inv, dyuv2inv, nuvisc;
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
template <bool SG>
__device__ __forceinline__ float face_flux_geo(const ScnDev& S, const StepVals& st, int dir, bool adv_on,
                                               bool theta_on, const FaceGeo& geo, uint8_t kf, float zs_nm,
                                               float zs_nmu, float hu, float gnavg2, float phi, const FaceV& a,
                                               bool dry_nm, bool dry_nmu, float zd_nm, float zd_nmu, float& q_out,
                                               float& uv_out) {
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
      frc = frc + S.fcorio * hu * a.vu;
    else
      frc = frc - S.fcorio * hu * a.vu;
  }
  if (S.wind) {
    const float tauw = dir == 0 ? st.twu : st.twv;
    const float hwet = hu / phi;
    if (hwet > 0.25f)
      frc = frc + phi * tauw;
    else
      frc = frc + tauw * hu * 4.0f;
  }
  float qfr;
  if (!(kf & KF_WET)) {
    qfr = sqrtf(fabsf(dzdx) / (fmaxf(gnavg2, 1.0e-5f) / 10.0f)) * powf(hu, 5.0f / 3.0f);
  } else if (S.friction2d) {
    qfr = sqrtf(a.qx_nm * a.qx_nm + (hu * a.vu) * (hu * a.vu));
  } else {
    qfr = fabsf(a.qx_nm);
  }
  float qsm = a.qx_nm;
  if (S.thetasmooth && theta_on && fabsf(a.qx_nmd) > 1.0e-6f && fabsf(a.qx_nmu) > 1.0e-6f)
    qsm = S.theta * a.qx_nm + 0.5f * (1.0f - S.theta) * (a.qx_nmu + a.qx_nmd);
  const float dt = st.dt;
  // hu**2 * hu**(1.0/3.0) (:673).  The real*4 exponent 1.0/3.0 is 0.333333343,
  // so hu**expo and cbrt(hu) differ by a factor hu**(1e-8): under one ulp for
  // 1e-3 <= hu <= 1e3.  cbrtf is the cheaper of the two on the device.
  const float hu73 = hu * hu * cbrtf(hu);
  float q = (qsm + frc * dt) / (1.0f + gnavg2 * dt * qfr / hu73);
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
