// B200 kernels of the SFINCS time-stepping core (sm_100a).
//
// One model time step is three launches (four with point sources), all driven
// by a device-resident table of scenarios so that one launch advances one model
// (BMI drop-in) or an uneven ensemble:
//
//   k_step_bnd      one CTA per scenario: dt = alfa*min_dt, t += dt (FP64),
//                   uniform meteo and boundary time interpolation, water-level
//                   boundary cells and weakly-reflective boundary fluxes.
//                   Restates sfincs_lib.f90:379-548, sfincs_meteo.f90:1445-1558,
//                   sfincs_boundaries.f90:682-1122.
//   k_momentum<SG>  one thread per cell, both owned faces (right u, upper v):
//                   local-inertia flux update, subgrid uv lookup, advection,
//                   viscosity, Coriolis, wind, friction, limiters; block min of
//                   the CFL time step and ONE atomicMin per CTA.
//                   Restates sfincs_momentum.f90:157-752.
//   k_sources       point sources, sequential like the reference (only if any).
//                   sfincs_continuity.f90:87-106, 311-325.
//   k_continuity<SG> one thread per cell: flux divergence, rain/infiltration/
//                   qext, subgrid volume -> level inversion, wiggle derivative,
//                   zsmax.  sfincs_continuity.f90:46-262, 265-624.
//
// The kernels are HBM-bound stencils (~0.2 flop/byte): no tensor-core work.
// Float expressions are written in the reference's evaluation order and the
// library is compiled with -fmad=false, so results round like the Fortran.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "sfg_device.h"

namespace sfg {

__device__ __forceinline__ float warp_min(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int64_t off(const ScnDev& S, int n, int m) {
  return (int64_t)m * S.ld + kGhostPad + n;
}

// --------------------------------------------------------------------------
// Step control + boundary forcing: one CTA per scenario.
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_step_bnd(const ScnDev* __restrict__ scns) {
  const ScnDev& S = scns[blockIdx.x];
  StepState& st = *S.st;
  __shared__ int s_go, s_itb0, s_itb1;
  __shared__ float s_tbfac;
  __shared__ double s_red[16];
  if (threadIdx.x == 0) {
    if (st.run) {  // previous step executed: its outputs are in the other buffer
      st.parity ^= 1;
      st.run = 0;
    }
    if (st.stop_pending) {  // sfincs_lib.f90:646
      st.t = (double)S.t1 + 1.0;
      st.stop_pending = 0;
    }
    int go = (st.t < st.tend) && (st.steps_left != 0);
    if (go) {
      st.nt += 1;
      float mdt = __uint_as_float(st.min_dt_bits);
      float dt = S.alfa * mdt;  // sfincs_lib.f90:391-392
      float dtchk = S.alfa * mdt;
      st.min_dt = mdt;
      st.dt = dt;
      double t = st.t + (double)dt;
      st.t = t;
      // ---- uniform wind from time series (sfincs_meteo.f90:1445-1508)
      if (S.wind) {
        for (int itw = st.itwndlast; itw <= S.ntwnd; itw++) {
          if ((double)S.twnd[itw - 1] > t) {
            int i0 = itw - 1 >= 1 ? itw - 1 : 1;
            float twfac = (float)((t - (double)S.twnd[i0 - 1]) / (double)(S.twnd[itw - 1] - S.twnd[i0 - 1]));
            float vmag = S.wmag[i0 - 1] * (1.0f - twfac) + S.wmag[itw - 1] * twfac;
            float twopi = 2.0f * S.pi;
            float dr0 = fmodf(S.wdir[i0 - 1], twopi);
            if (dr0 < 0.0f) dr0 += twopi;
            float dr1 = fmodf(S.wdir[itw - 1], twopi);
            if (dr1 < 0.0f) dr1 += twopi;
            if (dr1 > dr0 + S.pi)
              dr0 = dr0 + 2.0f * S.pi;
            else if (dr0 > dr1 + S.pi)
              dr1 = dr1 + 2.0f * S.pi;
            float vdir = dr0 * (1.0f - twfac) + dr1 * twfac;
            int icd = (int)(vmag * 10.0f) + 1;
            icd = icd < 1 ? 1 : (icd > 1000 ? 1000 : icd);
            float cd = S.cdval[icd - 1];
            st.twu = vmag * vmag * cosf(vdir) * S.rhoa * cd / S.rhow;
            st.twv = vmag * vmag * sinf(vdir) * S.rhoa * cd / S.rhow;
            st.itwndlast = itw - 1 >= 1 ? itw - 1 : 1;
            break;
          }
        }
      }
      // ---- uniform rain from time series (sfincs_meteo.f90:1510-1558)
      if (S.precip) {
        int itp;
        for (itp = st.itprcplast; itp <= S.ntprcp; itp++)
          if ((double)S.tprcp[itp - 1] > t) break;
        itp = max(min(itp, S.ntprcp), 1);
        int i0 = itp - 1 >= 1 ? itp - 1 : 1;
        float twfac = (i0 == itp) ? 0.0f
                                  : (float)((t - (double)S.tprcp[i0 - 1]) / (double)(S.tprcp[itp - 1] - S.tprcp[i0 - 1]));
        st.ptmp = (S.vprcp[i0 - 1] * (1.0f - twfac) + S.vprcp[itp - 1] * twfac) / (float)(1000 * 3600);
        st.itprcplast = itp - 1 >= 1 ? itp - 1 : 1;
      }
      // ---- boundary time interpolation (sfincs_boundaries.f90:696-726)
      int itb0 = 1, itb1 = 1;
      float tb = 0.0f;
      if (S.nbnd > 0) {
        if ((double)S.t_bnd[0] > (t - 1.0e-3)) {
          itb0 = itb1 = 1;
          tb = S.t_bnd[0];
        } else if ((double)S.t_bnd[S.ntbnd - 1] < (t + 1.0e-3)) {
          itb0 = itb1 = S.ntbnd;
          tb = S.t_bnd[S.ntbnd - 1];
        } else {
          for (int itb = st.itbndlast; itb <= S.ntbnd; itb++) {
            if ((double)S.t_bnd[itb - 1] > (t + 1.0e-6)) {
              itb0 = itb - 1;
              itb1 = itb;
              tb = (float)t;
              st.itbndlast = itb - 1;
              break;
            }
          }
        }
        s_tbfac = (tb - S.t_bnd[itb0 - 1]) / fmaxf(S.t_bnd[itb1 - 1] - S.t_bnd[itb0 - 1], 1.0e-6f);
      }
      s_itb0 = itb0;
      s_itb1 = itb1;
      st.min_dt_bits = __float_as_uint(S.dtmax);  // sfincs_momentum.f90:99
      if (dtchk < S.dtmin && st.nt > 1) {         // sfincs_lib.f90:634-648
        st.error = 1;
        st.stop_pending = 1;
      }
      st.run = 1;
      if (st.steps_left > 0) st.steps_left -= 1;
      if (S.precip) st.rain_vol += (double)st.ptmp * (double)S.area * (double)dt;
    }
    s_go = go;
  }
  __syncthreads();
  if (!s_go) return;
  const float dt = st.dt;
  const double t = st.t;
  const int p = st.parity;
  // ---- boundary point levels zst_bnd (sfincs_boundaries.f90:728-756)
  for (int ib = threadIdx.x; ib < S.nbnd; ib += blockDim.x) {
    const float* z0 = S.zs_bnd + (size_t)(s_itb0 - 1) * S.nbnd;
    const float* z1 = S.zs_bnd + (size_t)(s_itb1 - 1) * S.nbnd;
    S.zst_bnd[ib] = z0[ib] + (z1[ib] - z0[ib]) * s_tbfac;
  }
  // ---- point-source discharges (sfincs_discharges.f90:341-359)
  if (S.nsrc > 0 && threadIdx.x == 0) {
    for (int its = st.itsrclast; its <= S.ntsrc; its++) {
      if ((double)S.tsrc[its - 1] > t) {
        int i0 = its - 1 >= 1 ? its - 1 : 1;
        const float* a = S.qsrc + (size_t)(i0 - 1) * S.nsrc;
        const float* b = S.qsrc + (size_t)(its - 1) * S.nsrc;
        for (int is = 0; is < S.nsrc; is++)
          S.qtsrc[is] = (float)((double)a[is] + (double)(b[is] - a[is]) * (t - (double)S.tsrc[i0 - 1]) /
                                                    (double)(S.tsrc[its - 1] - S.tsrc[i0 - 1]));
        st.itsrclast = its - 1 >= 1 ? its - 1 : 1;
        break;
      }
    }
  }
  __syncthreads();
  // ---- boundary cells: water levels and Neumann copies (sfincs_boundaries.f90:789-917)
  for (int ib = threadIdx.x; ib < S.ngbnd; ib += blockDim.x) {
    const int8_t k = S.gb_kcs[ib];
    const int nmb = S.gb_cell[ib];
    if (k == 2 && S.nbnd > 0) {
      double zst;
      if (S.nbnd > 1)
        zst = (double)(S.zst_bnd[S.gb_i1[ib]] * S.gb_fac[ib] + S.zst_bnd[S.gb_i2[ib]] * (1.0f - S.gb_fac[ib]));
      else
        zst = (double)S.zst_bnd[0];
      float zb0, zb1;
      if (t < (double)(S.tspinup - 1.0e-3f)) {
        float smfac = (float)(1.0 - (t - (double)S.t0) / (double)(S.tspinup - S.t0));
        float zs0act = (float)zst;
        zb0 = S.zini * smfac + zs0act * (1.0f - smfac);
        zb1 = zb0;
      } else {
        zb0 = (float)zst;
        zb1 = (float)zst;
      }
      const float floor_z = S.subgrid ? S.zz_min[nmb] : S.zb[nmb];
      S.zsb0[ib] = fmaxf(zb0, floor_z);
      S.zsb[ib] = fmaxf(zb1, floor_z);
    } else if (k == 6) {
      S.zs[nmb] = S.zs[S.gb_nmi[ib]];
    }
  }
  __syncthreads();
  // ---- weakly reflective boundary fluxes at kcuv==2 faces (sfincs_boundaries.f90:941-1120)
  const float factime = fminf(dt / S.btfilter, 1.0f);
  const float one_minus_factime = 1.0f - factime;
  const float facrel = 1.0f - fminf(dt / S.btrelax, 1.0f);
  double inflow = 0.0;
  for (int ib = threadIdx.x; ib < S.nkcuv2; ib += blockDim.x) {
    const int ip = S.kb_face[ib];
    const int dir = S.kb_dir[ib];
    const int indb = S.kb_gb[ib];
    const int nmb = S.gb_cell[indb];
    const int nmi = S.kb_nmi[ib];
    const float sgn = (float)S.kb_sign[ib];
    float zsnmi = S.zs[nmi];
    float zsnmb = S.zsb[indb];
    float zs0nmb = S.zsb0[indb];
    float hnmb;
    if (S.subgrid) {
      const float2 zr = dir == 0 ? S.sgz_u[ip] : S.sgz_v[ip];
      const float zsuv = fmaxf(zsnmb, zsnmi);
      float depthuv;
      if (zsuv >= zr.y - 1.0e-4f) {
        depthuv = (dir == 0 ? S.sgw_u[ip] : S.sgw_v[ip]).x + zsuv;
      } else if (zsuv > zr.x) {
        float dzuv = (zr.y - zr.x) / (float)(S.nlev - 1);
        int iuv = (int)((zsuv - zr.x) / dzuv) + 1;
        float facint = (zsuv - (zr.x + (float)(iuv - 1) * dzuv)) / dzuv;
        const UvRec r = (dir == 0 ? S.rec_u : S.rec_v)[(int64_t)(iuv - 1) * S.nalloc + ip];
        depthuv = r.havg + r.dhavg * facint;
      } else {
        depthuv = 0.0f;
      }
      hnmb = fmaxf(depthuv, S.huthresh);
      zsnmb = fmaxf(zsnmb, S.zz_min[nmb]);
      zs0nmb = fmaxf(zs0nmb, S.zz_min[nmb]);
    } else {
      hnmb = fmaxf(0.5f * (zsnmb + zsnmi) - S.kb_zbuv[ib], S.huthresh);
      zsnmb = fmaxf(zsnmb, S.zb[nmb]);
      zs0nmb = fmaxf(zs0nmb, S.zb[nmb]);
    }
    float qq, uu;
    float* qa = dir == 0 ? S.qu[p] : S.qv[p];
    float* qb = dir == 0 ? S.qu[p ^ 1] : S.qv[p ^ 1];
    float* ua = dir == 0 ? S.uu[p] : S.vv[p];
    float* ub_ = dir == 0 ? S.uu[p ^ 1] : S.vv[p ^ 1];
    if (hnmb < S.huthresh + 1.0e-6f) {
      qq = 0.0f;
      uu = 0.0f;
      S.uvmean[ib] = 0.0f;
    } else {
      const float sq = sqrtf(S.g / hnmb);
      const float ui = sq * (zsnmb - zs0nmb);
      const float ubv = sgn * (2.0f * ui - sq * (zsnmi - zs0nmb));
      qq = ubv * hnmb + S.uvmean[ib];
      if (S.subgrid) {
        if (S.zvol[nmi] <= 0.0) qq = sgn > 0.0f ? fmaxf(qq, 0.0f) : fminf(qq, 0.0f);
        if (zsnmb - S.zz_min[nmb] < S.huthresh) qq = sgn > 0.0f ? fminf(qq, 0.0f) : fmaxf(qq, 0.0f);
      } else {
        if (zsnmi - S.zb[nmi] <= S.huthresh) qq = sgn > 0.0f ? fmaxf(qq, 0.0f) : fminf(qq, 0.0f);
        if (zsnmb - S.zb[nmb] < S.huthresh) qq = sgn > 0.0f ? fminf(qq, 0.0f) : fmaxf(qq, 0.0f);
      }
      uu = fmaxf(fminf(qq / hnmb, 4.0f), -4.0f);
    }
    qa[ip] = qq;
    qb[ip] = qq;
    ua[ip] = uu;
    ub_[ip] = uu;
    if (S.btfilter >= -1.0e-6f)
      S.uvmean[ib] = factime * qq + facrel * one_minus_factime * S.uvmean[ib];
    else
      S.uvmean[ib] = 0.0f;
    const float zsb_v = S.zsb[indb];
    S.zs[nmb] = zsb_v;
    if (S.store_zsmax) S.zsmax[nmb] = fmaxf(S.zsmax[nmb], zsb_v);
    inflow += (double)sgn * (double)qq * (double)(dir == 0 ? S.dy : S.dx) * (double)dt;
  }
  // FP64 volume-balance accumulator for the boundary inflow (fixed-order block reduction)
  inflow = warp_sum(inflow);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = inflow;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += s_red[w];
    st.bflux_vol += tot;
  }
}

// --------------------------------------------------------------------------
// Momentum: one face update (shared by u and v faces).
// --------------------------------------------------------------------------
struct FaceNb {
  float zs_nm, zs_nmu;
  float qx_nm, qx_nmd, qx_nmu, qy_nm, qy_nmu, qy_ndm, qy_ndmu;
  float uu_nm, uu_nmd, uu_nmu, uu_ndm, uu_num, vu;
  float dxuvinv, dyuvinv, dxuv2inv, dyuv2inv;
  float tauw;
  bool adv_on, theta_ok, was_wet, is_v;
};

struct FaceSg {  // subgrid depth/roughness lookups, or regular-grid values
  float hu, gnavg2, phi;
};

template <bool SG>
__device__ __forceinline__ void face_update(const ScnDev& S, const FaceNb& a, const FaceSg& d, float dt, bool nm_dry,
                                            bool nmu_dry, float zsderv_nm, float zsderv_nmu, float& q_out,
                                            float& uv_out, float& mdt) {
  const float hu = d.hu;
  const float gnavg2 = d.gnavg2;
  const float phi = d.phi;
  const float hwet = hu / phi;
  float dzdx;
  if (S.slopelim < 9999.0f)
    dzdx = fminf(fmaxf((a.zs_nmu - a.zs_nm) * a.dxuvinv, -S.slopelim), S.slopelim);
  else
    dzdx = (a.zs_nmu - a.zs_nm) * a.dxuvinv;
  float frc = -S.g * hu * dzdx;
  if (S.advection && a.adv_on) {
    float dqxudx = 0.0f, dqyudy = 0.0f;
    if (S.adv_scheme == 0) {
      if (a.qx_nm > 1.0e-6f)
        dqxudx = (a.qx_nm * a.uu_nm - a.qx_nmd * a.uu_nmd) * a.dxuvinv;
      else if (a.qx_nm < -1.0e-6f)
        dqxudx = (a.qx_nmu * a.uu_nmu - a.qx_nm * a.uu_nm) * a.dxuvinv;
      const float qy = a.qy_ndm + a.qy_ndmu + a.qy_nm + a.qy_nmu;
      if (qy > 1.0e-6f)
        dqyudy = (a.qy_ndm + a.qy_ndmu) * (a.uu_nm - a.uu_ndm) * a.dyuvinv / 2.0f;
      else if (qy < -1.0e-6f)
        dqyudy = (a.qy_nm + a.qy_nmu) * (a.uu_num - a.uu_nm) * a.dyuvinv / 2.0f;
    } else {
      float qd = (a.qx_nmd + a.qx_nm) / 2.0f;
      float qu = (a.qx_nm + a.qx_nmu) / 2.0f;
      if (qd > 1.0e-6f) {
        const float ud = (a.uu_nmd + a.uu_nm) / 2.0f;
        dqxudx = (qd * (a.uu_nm - a.uu_nmd) + ud * (a.qx_nm - a.qx_nmd)) * a.dxuvinv;
      }
      if (qu < -1.0e-6f) {
        const float uu = (a.uu_nm + a.uu_nmu) / 2.0f;
        dqxudx = dqxudx + (qu * (a.uu_nmu - a.uu_nm) + uu * (a.qx_nmu - a.qx_nm)) * a.dxuvinv;
      }
      qu = (a.qy_nm + a.qy_nmu) / 2.0f;
      qd = (a.qy_ndm + a.qy_ndmu) / 2.0f;
      if (qd > 1.0e-6f) dqyudy = qd * (a.uu_nm - a.uu_ndm) * a.dyuvinv;
      if (qu < -1.0e-6f) dqyudy = dqyudy + qu * (a.uu_num - a.uu_nm) * a.dyuvinv;
      const float ud = (a.uu_nmd + a.uu_nm) / 2.0f;
      const float uu = (a.uu_nm + a.uu_nmu) / 2.0f;
      if (ud > 1.0e-6f) dqyudy = dqyudy + ud * (a.qy_nm - a.qy_ndm) * a.dyuvinv;
      if (uu < -1.0e-6f) dqyudy = dqyudy + uu * (a.qy_nmu - a.qy_ndmu) * a.dyuvinv;
    }
    float adv = -phi * (dqxudx + dqyudy);
    adv = fminf(fmaxf(adv, -S.advlim * hu), S.advlim * hu);
    frc = frc + adv;
  }
  if (S.viscosity) {
    frc = frc + S.nuvisc * hu *
                    ((a.uu_nmu - 2.0f * a.uu_nm + a.uu_nmd) * a.dxuv2inv +
                     (a.uu_num - 2.0f * a.uu_nm + a.uu_ndm) * a.dyuv2inv);
  }
  if (S.coriolis) {  // sfincs_momentum.f90:533-545
    if (!a.is_v)
      frc = frc + S.fcorio * hu * a.vu;
    else
      frc = frc - S.fcorio * hu * a.vu;
  }
  if (S.wind) {
    if (hwet > 0.25f)
      frc = frc + phi * a.tauw;
    else
      frc = frc + a.tauw * hu * 4.0f;
  }
  float qfr;
  if (!a.was_wet) {
    qfr = sqrtf(fabsf(dzdx) / (fmaxf(gnavg2, 1.0e-5f) / 10.0f)) * powf(hu, 5.0f / 3.0f);
  } else if (S.friction2d) {
    qfr = sqrtf(a.qx_nm * a.qx_nm + (hu * a.vu) * (hu * a.vu));
  } else {
    qfr = fabsf(a.qx_nm);
  }
  float qsm = a.qx_nm;
  if (S.thetasmooth && a.theta_ok && fabsf(a.qx_nmd) > 1.0e-6f && fabsf(a.qx_nmu) > 1.0e-6f)
    qsm = S.theta * a.qx_nm + 0.5f * (1.0f - S.theta) * (a.qx_nmu + a.qx_nmd);
  const float hu73 = hu * hu * powf(hu, 1.0f / 3.0f);
  float q = (qsm + frc * dt) / (1.0f + gnavg2 * dt * qfr / hu73);
  if (SG && S.wiggle) {
    const float mdrv = fabsf(zsderv_nm - zsderv_nmu) - S.wiggle_threshold;
    if (mdrv > 0.0f) q = q * S.wiggle_threshold / (S.wiggle_factor * mdrv + S.wiggle_threshold);
  }
  if (nm_dry) q = fminf(q, 0.0f);
  if (nmu_dry) q = fmaxf(q, 0.0f);
  q = fminf(fmaxf(q, -hu * S.uvlim), hu * S.uvlim);
  const float uv = q / fmaxf(hu, S.huvmin);
  q_out = q;
  uv_out = uv;
  const float min_dt_ip = 1.0f / (fmaxf(sqrtf(S.g * hu), fabsf(uv)) * a.dxuvinv);
  mdt = fminf(mdt, min_dt_ip);
}

template <bool SG>
__device__ __forceinline__ bool face_depth(const ScnDev& S, int dir, int64_t c, float zsu, FaceSg& d) {
  if (SG) {
    const float2 zr = dir == 0 ? S.sgz_u[c] : S.sgz_v[c];
    const float zmin = zr.x, zmax = zr.y;
    if (!(zsu > zmin + S.huthresh)) return false;
    d.phi = 1.0f;
    if (zsu > zmax) {
      const float4 w = dir == 0 ? S.sgw_u[c] : S.sgw_v[c];
      d.hu = w.x + zsu;
      d.gnavg2 = w.z - (w.z - w.y) / (w.w * (zsu - zmax) + 1.0f);
    } else {
      const float dzuv = (zmax - zmin) / (float)(S.nlev - 1);
      int iuv = (int)((zsu - zmin) / dzuv) + 1;
      iuv = min(iuv, S.nlev - 1);
      const float facint = (zsu - (zmin + (float)(iuv - 1) * dzuv)) / dzuv;
      const UvRec r = (dir == 0 ? S.rec_u : S.rec_v)[(int64_t)(iuv - 1) * S.nalloc + c];
      d.hu = r.havg + r.dhavg * facint;
      d.gnavg2 = r.nrep + r.dnrep * facint;
      d.phi = r.pwet + r.dpwet * facint;
    }
    return true;
  } else {
    const float zbmx = dir == 0 ? S.zbmx_u[c] : S.zbmx_v[c];
    if (!(zsu > zbmx)) return false;
    d.hu = fmaxf(zsu - zbmx, S.huthresh);
    d.gnavg2 = dir == 0 ? S.gn2_u[c] : S.gn2_v[c];
    d.phi = 1.0f;
    return true;
  }
}

template <bool SG>
__global__ void __launch_bounds__(256) k_momentum(const ScnDev* __restrict__ scns, const Tile* __restrict__ tiles) {
  const Tile tl = tiles[blockIdx.x];
  const ScnDev& S = scns[tl.scn];
  const StepState& st = *S.st;
  if (!st.run) return;
  const int p = st.parity;
  const float dt = st.dt;
  const int n = tl.n0 + threadIdx.x;
  const int m = tl.m0 + threadIdx.y;
  float mdt = FLT_MAX;
  if (n <= S.nmax && m <= S.mmax) {
    const int64_t c = off(S, n, m);
    const int64_t ld = S.ld;
    const uint16_t f = S.flags[c];
    const float* __restrict__ qu0 = S.qu[p];
    const float* __restrict__ qv0 = S.qv[p];
    const float* __restrict__ uu0 = S.uu[p];
    const float* __restrict__ vv0 = S.vv[p];
    uint8_t kf = S.kfuv[c];
    const uint8_t kf_old = kf;
    const float zs_c = S.zs[c];
    float zd_c = 0.0f;
    bool dry_c = false;
    if (f & (F_UACT | F_VACT)) {
      if (SG) {
        zd_c = S.wiggle ? S.zsderv[c] : 0.0f;
        dry_c = S.vneg[c] != 0;
      } else {
        dry_c = zs_c < S.zb[c];
      }
    }
    if (f & F_UACT) {  // ---------------- u face: (n,m) -> (n,m+1)
      FaceNb a;
      a.zs_nm = zs_c;
      a.zs_nmu = S.zs[c + ld];
      const float zsu = fmaxf(a.zs_nm, a.zs_nmu);
      FaceSg d;
      float qn = 0.0f, un = 0.0f;
      if (face_depth<SG>(S, 0, c, zsu, d)) {
        a.dxuvinv = S.dxinv;
        a.dyuvinv = S.dyinv;
        a.dxuv2inv = S.dx2inv;
        a.dyuv2inv = S.dy2inv;
        a.qx_nm = qu0[c];
        a.qx_nmd = qu0[c - ld];
        a.qx_nmu = qu0[c + ld];
        a.qy_nm = qv0[c];
        a.qy_nmu = qv0[c + ld];
        a.qy_ndm = qv0[c - 1];
        a.qy_ndmu = qv0[c + ld - 1];
        a.uu_nm = uu0[c];
        a.uu_nmd = uu0[c - ld];
        a.uu_nmu = uu0[c + ld];
        a.uu_ndm = (f & F_CDN) ? uu0[c - 1] : a.uu_nm;
        a.uu_num = (f & F_CUP) ? uu0[c + 1] : a.uu_nm;
        a.vu = (vv0[c - 1] + vv0[c + ld - 1] + vv0[c] + vv0[c + ld]) / 4.0f;
        a.tauw = st.twu;
        a.adv_on = (f & F_UADV) != 0;
        a.theta_ok = (f & F_UTH) != 0;
        a.was_wet = (kf_old & K_U) != 0;
        a.is_v = false;
        bool dry_u;
        float zd_u = 0.0f;
        if (SG) {
          dry_u = S.vneg[c + ld] != 0;
          zd_u = S.wiggle ? S.zsderv[c + ld] : 0.0f;
        } else {
          dry_u = a.zs_nmu < S.zb[c + ld];
        }
        face_update<SG>(S, a, d, dt, dry_c, dry_u, zd_c, zd_u, qn, un, mdt);
        kf |= K_U;
      } else {
        kf &= (uint8_t)~K_U;
      }
      S.qu[p ^ 1][c] = qn;
      S.uu[p ^ 1][c] = un;
    }
    if (f & F_VACT) {  // ---------------- v face: (n,m) -> (n+1,m)
      FaceNb a;
      a.zs_nm = zs_c;
      a.zs_nmu = S.zs[c + 1];
      const float zsu = fmaxf(a.zs_nm, a.zs_nmu);
      FaceSg d;
      float qn = 0.0f, un = 0.0f;
      if (face_depth<SG>(S, 1, c, zsu, d)) {
        a.dxuvinv = S.dyinv;
        a.dyuvinv = S.dxinv;
        a.dxuv2inv = S.dy2inv;
        a.dyuv2inv = S.dx2inv;
        a.qx_nm = qv0[c];
        a.qx_nmd = qv0[c - 1];
        a.qx_nmu = qv0[c + 1];
        a.qy_nm = qu0[c];
        a.qy_nmu = qu0[c + 1];
        a.qy_ndm = qu0[c - ld];
        a.qy_ndmu = qu0[c + 1 - ld];
        a.uu_nm = vv0[c];
        a.uu_nmd = vv0[c - 1];
        a.uu_nmu = vv0[c + 1];
        a.uu_ndm = (f & F_CLF) ? vv0[c - ld] : a.uu_nm;
        a.uu_num = (f & F_CRT) ? vv0[c + ld] : a.uu_nm;
        a.vu = (uu0[c - ld] + uu0[c + 1 - ld] + uu0[c] + uu0[c + 1]) / 4.0f;
        a.tauw = st.twv;
        a.adv_on = (f & F_VADV) != 0;
        a.theta_ok = (f & F_VTH) != 0;
        a.was_wet = (kf_old & K_V) != 0;
        a.is_v = true;
        bool dry_u;
        float zd_u = 0.0f;
        if (SG) {
          dry_u = S.vneg[c + 1] != 0;
          zd_u = S.wiggle ? S.zsderv[c + 1] : 0.0f;
        } else {
          dry_u = a.zs_nmu < S.zb[c + 1];
        }
        face_update<SG>(S, a, d, dt, dry_c, dry_u, zd_c, zd_u, qn, un, mdt);
        kf |= K_V;
      } else {
        kf &= (uint8_t)~K_V;
      }
      S.qv[p ^ 1][c] = qn;
      S.vv[p ^ 1][c] = un;
    }
    if (kf != kf_old) S.kfuv[c] = kf;
  }
  // CTA min of the CFL time step, then one atomicMin per CTA (float bits of a positive value)
  __shared__ float s_min[8];
  mdt = warp_min(mdt);
  const int lane = threadIdx.x, warp = threadIdx.y;
  if (lane == 0) s_min[warp] = mdt;
  __syncthreads();
  if (warp == 0) {
    float v = lane < (int)blockDim.y ? s_min[lane] : FLT_MAX;
    v = warp_min(v);
    if (lane == 0 && v < FLT_MAX) atomicMin(&S.st->min_dt_bits, __float_as_uint(v));
  }
}

// --------------------------------------------------------------------------
// Point sources, applied in the reference's sequential order before the cell loop.
// --------------------------------------------------------------------------
__global__ void k_sources(const ScnDev* __restrict__ scns) {
  const ScnDev& S = scns[blockIdx.x];
  StepState& st = *S.st;
  if (!st.run || S.nsrc == 0 || threadIdx.x != 0) return;
  const float dt = st.dt;
  double vol = 0.0;
  for (int is = 0; is < S.nsrc; is++) {
    const int c = S.src_cell[is];
    if (S.subgrid) {
      if (S.zvol[c] >= 0.0) {
        S.zvol[c] = S.zvol[c] + (double)(S.qtsrc[is] * dt);
        vol += (double)(S.qtsrc[is] * dt);
      }
    } else {
      const float before = S.zs[c];
      const float z = fmaxf(S.zs[c] + S.qtsrc[is] * dt / S.area, S.zb[c]);
      S.zs[c] = z;
      vol += ((double)z - (double)before) * (double)S.area;
    }
  }
  st.src_vol += vol;
}

// --------------------------------------------------------------------------
// Continuity.
// --------------------------------------------------------------------------
template <bool SG>
__global__ void __launch_bounds__(256) k_continuity(const ScnDev* __restrict__ scns, const Tile* __restrict__ tiles) {
  const Tile tl = tiles[blockIdx.x];
  const ScnDev& S = scns[tl.scn];
  const StepState& st = *S.st;
  if (!st.run) return;
  const int n = tl.n0 + threadIdx.x;
  const int m = tl.m0 + threadIdx.y;
  if (n > S.nmax || m > S.mmax) return;
  const int64_t c = off(S, n, m);
  const uint16_t f = S.flags[c];
  if (!(f & F_ACT)) return;
  const int p1 = st.parity ^ 1;  // buffers written by this step's momentum
  const float dt = st.dt;
  float zsn;
  if (f & F_KCS1) {
    const float* __restrict__ qu = S.qu[p1];
    const float* __restrict__ qv = S.qv[p1];
    const int64_t ld = S.ld;
    const float q_md = qu[c - ld], q_mu = qu[c], q_nd = qv[c - 1], q_nu = qv[c];
    if (SG) {
      const double v_old = S.zvol[c];
      float dvol = ((q_md - q_mu) * S.dy + (q_nd - q_nu) * S.dx) * dt;
      if (S.precip || S.use_qext) {
        float dzsdt = 0.0f;
        if (S.precip) {
          float qinfmap = 0.0f;
          if (S.infiltration) qinfmap = v_old <= 0.0 ? 0.0f : S.qinf[c];
          dzsdt = dzsdt + (st.ptmp - qinfmap);
        }
        if (S.use_qext) dzsdt = dzsdt + S.qext[c];
        dvol = dvol + dzsdt * S.area * dt;
      }
      const double v = v_old + (double)dvol;
      S.zvol[c] = v;
      float zs00 = 0.0f, zs11 = 0.0f;
      if (S.wiggle) {
        zs00 = S.zs0[c];
        zs11 = S.zs[c];
        S.zs0[c] = zs11;
      }
      const float volmax = S.zz_volmax[c];
      if (v >= (double)(volmax * 0.999f)) {
        zsn = (float)((double)fmaxf(S.zz_max[c], -20.0f) + (v - (double)volmax) / (double)S.area);
      } else if (v <= (double)1.0e-6f) {
        zsn = fmaxf(S.zz_min[c], -20.0f);
      } else {
        const float dzvol = volmax / (float)(S.nlev - 1);
        const int iuv = (int)(v / (double)dzvol) + 1;
        const float facint = (float)((v - (double)((float)(iuv - 1) * dzvol)) / (double)dzvol);
        const float2 dep = S.zlev[(int64_t)(iuv - 1) * S.nalloc + c];
        zsn = dep.x + dep.y * facint;
      }
      S.zs[c] = zsn;
      if (S.wiggle) S.zsderv[c] = zsn - 2.0f * zs11 + zs00;
      S.vneg[c] = v < 0.0 ? 1 : 0;
    } else {
      float z = S.zs[c];
      if (S.precip) {
        float qinfmap = 0.0f;
        if (S.infiltration) qinfmap = z <= S.zb[c] ? 0.0f : S.qinf[c];
        z = z + (st.ptmp - qinfmap) * dt;
      }
      if (S.use_qext) z = z + S.qext[c] * dt;
      z = z + ((q_md - q_mu) * S.dxinv + (q_nd - q_nu) * S.dyinv) * dt;
      S.zs[c] = z;
      zsn = z;
    }
  } else {
    zsn = S.zs[c];
  }
  if (S.store_zsmax) {
    const float zm = S.zsmax[c];
    if (zsn > zm) S.zsmax[c] = zsn;
  }
}

// --------------------------------------------------------------------------
// Host-callable launchers (C linkage inside the library only).
// --------------------------------------------------------------------------
void launch_step(const ScnDev* d_scns, int nscn, const Tile* d_tiles, int ntiles, int subgrid, int any_src,
                 cudaStream_t s) {
  k_step_bnd<<<nscn, 512, 0, s>>>(d_scns);
  dim3 blk(32, 8);
  if (ntiles > 0) {
    if (subgrid)
      k_momentum<true><<<ntiles, blk, 0, s>>>(d_scns, d_tiles);
    else
      k_momentum<false><<<ntiles, blk, 0, s>>>(d_scns, d_tiles);
  }
  if (any_src) k_sources<<<nscn, 32, 0, s>>>(d_scns);
  if (ntiles > 0) {
    if (subgrid)
      k_continuity<true><<<ntiles, blk, 0, s>>>(d_scns, d_tiles);
    else
      k_continuity<false><<<ntiles, blk, 0, s>>>(d_scns, d_tiles);
  }
}

}  // namespace sfg
