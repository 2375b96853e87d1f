// B200 kernels of the SFINCS time-stepping core (sm_100a).
//
// One model time step is three launches (four with point sources), all driven
// by a device-resident table of scenarios so that one launch advances one model
// (BMI drop-in) or an uneven ensemble with per-scenario dt:
//
//   k_step_bnd      one CTA per scenario: step control (dt = alfa*min_dt,
//                   t += dt in FP64, uniform meteo, boundary time
//                   interpolation, CFL reset, instability check;
//                   sfincs_lib.f90:379-548, sfincs_meteo.f90:1445-1558,
//                   sfincs_boundaries.f90:682-758), then one thread per
//                   water-level boundary face / Neumann cell: boundary levels
//                   and weakly reflective fluxes (sfincs_boundaries.f90:761-1122).
//   k_momentum<SG>  one thread per uv face (blockDim.z selects u or v, warp
//                   uniform): local-inertia flux, subgrid uv lookup, advection,
//                   viscosity, Coriolis, wind, friction, limiters, and the CFL
//                   time step (CTA min + ONE atomicMin per CTA).
//                   sfincs_momentum.f90:157-752.
//   k_sources       point sources, sequential like the reference (only if any).
//                   sfincs_continuity.f90:87-106, 311-325.
//   k_continuity<SG> one thread per cell: flux divergence, rain/infiltration/
//                   qext, subgrid volume -> level inversion, wiggle derivative,
//                   zsmax.  sfincs_continuity.f90:46-262, 265-624.
//
// The path is an HBM-bound stencil plus table gathers (~0.2 flop/byte); there
// is no dense contraction, so no tensor-core work.  The kernels keep at most
// two dependent global-memory round trips per thread: every load whose address
// does not depend on loaded data is issued first (speculatively where the dense
// layout makes the address valid anyway), then one wave of data-dependent
// loads (neighbour fluxes of wet faces, table records).
// Float expressions follow the reference's evaluation order; the library is
// compiled with -fmad=false so they round like the Fortran and the oracle.
#include <cuda_runtime.h>

#include <algorithm>

#include <cfloat>
#include <cstdint>

#include "face_math.h"
#include "pdl.h"
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
// Step control.
// --------------------------------------------------------------------------
// What this step does, from the scenario's step state as the previous step left
// it.  Every thread of the step kernel computes it from the same loads, so the
// boundary work needs neither a barrier nor a round trip through memory after
// thread 0 decides the step; thread 0 then commits it (commit_step).
struct StepPlan {
  int go;          // the scenario takes this step
  int parity;      // buffer holding the latest q / uv after the step's turnover
  float mdt, dt;   // CFL time step of the previous step, this step's dt
  double t;        // model time after this step (the current time if !go)
  int itb0, itb1;  // boundary time records (1-based)
  int itbndlast;   // cached boundary time record for the next search
  float tbfac;     // boundary time-interpolation factor
  int meteo_upd;   // the gridded meteo window advances this step
  float mt0, mt1;  // the gridded meteo window of this step
};

__device__ __forceinline__ StepPlan plan_step(const ScnDev& S, const StepState& st) {
  StepPlan P;
  P.parity = st.run ? (st.parity ^ 1) : st.parity;  // previous step executed: its outputs are in the other buffer
  const double t_now = st.stop_pending ? (double)S.t1 + 1.0 : st.t;  // sfincs_lib.f90:646
  P.go = (t_now < st.tend) && (st.steps_left != 0);
  P.mdt = __uint_as_float(st.min_dt_bits);
  P.dt = S.alfa * P.mdt;  // sfincs_lib.f90:391-392
  P.t = P.go ? t_now + (double)P.dt : t_now;
  P.itbndlast = st.itbndlast;
  P.itb0 = st.itb0;
  P.itb1 = st.itb1;
  P.tbfac = st.tbfac;
  // ---- gridded meteo window (sfincs_lib.f90:493-503): t >= twindupd opens [twindupd, twindupd + dtwnd]
  P.meteo_upd = P.go && S.meteo3d && P.t >= (double)st.twindupd;
  P.mt0 = P.meteo_upd ? st.twindupd : st.meteo_t0;
  P.mt1 = P.meteo_upd ? st.twindupd + S.dtwnd : st.meteo_t1;
  // ---- boundary time interpolation (sfincs_boundaries.f90:696-726)
  if (P.go && S.nbnd > 0) {
    const double t = P.t;
    int itb0 = 1, itb1 = 1;
    float tb = 0.0f;
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
          P.itbndlast = itb - 1;
          break;
        }
      }
    }
    P.itb0 = itb0;
    P.itb1 = itb1;
    P.tbfac = (tb - S.t_bnd[itb0 - 1]) / fmaxf(S.t_bnd[itb1 - 1] - S.t_bnd[itb0 - 1], 1.0e-6f);
  }
  return P;
}

// Forcing of a step that goes: uniform wind and rain, point-source discharges.
// It writes only step-state fields that plan_step does not read, so one thread
// runs it while the others still derive the plan.
__device__ __forceinline__ void step_forcing(const ScnDev& S, StepState& st, const StepPlan& P) {
  const float dt = P.dt;
  const double t = P.t;
  // ---- uniform wind from time series (sfincs_meteo.f90:1445-1508)
  if (S.wind && S.ntwnd > 0) {
    for (int itw = st.itwndlast; itw <= S.ntwnd; itw++) {
      if ((double)S.twnd[itw - 1] > t) {
        const int i0 = itw - 1 >= 1 ? itw - 1 : 1;
        const float twfac = (float)((t - (double)S.twnd[i0 - 1]) / (double)(S.twnd[itw - 1] - S.twnd[i0 - 1]));
        const float vmag = S.wmag[i0 - 1] * (1.0f - twfac) + S.wmag[itw - 1] * twfac;
        const float twopi = 2.0f * S.pi;
        float dr0 = fmodf(S.wdir[i0 - 1], twopi);
        if (dr0 < 0.0f) dr0 += twopi;
        float dr1 = fmodf(S.wdir[itw - 1], twopi);
        if (dr1 < 0.0f) dr1 += twopi;
        if (dr1 > dr0 + S.pi)
          dr0 = dr0 + 2.0f * S.pi;
        else if (dr0 > dr1 + S.pi)
          dr1 = dr1 + 2.0f * S.pi;
        const float vdir = dr0 * (1.0f - twfac) + dr1 * twfac;
        int icd = (int)(vmag * 10.0f) + 1;
        icd = icd < 1 ? 1 : (icd > 1000 ? 1000 : icd);
        const float cd = S.cdval[icd - 1];
        st.twu = vmag * vmag * cosf(vdir) * S.rhoa * cd / S.rhow;
        st.twv = vmag * vmag * sinf(vdir) * S.rhoa * cd / S.rhow;
        st.itwndlast = itw - 1 >= 1 ? itw - 1 : 1;
        break;
      }
    }
  }
  // ---- uniform rain from time series (sfincs_meteo.f90:1510-1558)
  if (S.precip && S.ntprcp > 0) {
    int itp;
    for (itp = st.itprcplast; itp <= S.ntprcp; itp++)
      if ((double)S.tprcp[itp - 1] > t) break;
    itp = max(min(itp, S.ntprcp), 1);
    const int i0 = itp - 1 >= 1 ? itp - 1 : 1;
    const float twfac =
        (i0 == itp) ? 0.0f
                    : (float)((t - (double)S.tprcp[i0 - 1]) / (double)(S.tprcp[itp - 1] - S.tprcp[i0 - 1]));
    st.ptmp = (S.vprcp[i0 - 1] * (1.0f - twfac) + S.vprcp[itp - 1] * twfac) / (float)(1000 * 3600);
    st.itprcplast = itp - 1 >= 1 ? itp - 1 : 1;
    st.rain_vol += (double)st.ptmp * (double)dt;  // depth; the host multiplies by the kcs==1 area
  }
  // ---- point-source discharges (sfincs_discharges.f90:341-359)
  if (S.nsrc > 0) {
    for (int its = st.itsrclast; its <= S.ntsrc; its++) {
      if ((double)S.tsrc[its - 1] > t) {
        const int i0 = its - 1 >= 1 ? its - 1 : 1;
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
}

// Thread 0 writes the step's decisions and the rest of the step control (CFL
// reset, instability check) once no thread reads the step state any more.
__device__ __forceinline__ void commit_step(const ScnDev& S, StepState& st, const StepPlan& P) {
  if (st.run) {
    st.parity = P.parity;
    st.run = 0;
  }
  if (st.stop_pending) {  // sfincs_lib.f90:646
    st.t = (double)S.t1 + 1.0;
    st.stop_pending = 0;
  }
  if (!P.go) return;
  st.nt += 1;
  const float dtchk = S.alfa * P.mdt;
  st.min_dt = P.mdt;
  st.dt = P.dt;
  st.t = P.t;
  if (S.nbnd > 0) {
    st.itb0 = P.itb0;
    st.itb1 = P.itb1;
    st.tbfac = P.tbfac;
    st.itbndlast = P.itbndlast;
  }
  if (P.meteo_upd) {  // the gridded meteo window this step opened (the fields were made before this kernel)
    st.meteo_t0 = P.mt0;
    st.meteo_t1 = P.mt1;
    st.twindupd = st.twindupd + S.dtwnd;
  }
  st.min_dt_bits = __float_as_uint(S.dtmax);  // sfincs_momentum.f90:99
  if (dtchk < S.dtmin && st.nt > 1) {         // sfincs_lib.f90:634-648
    st.error = 1;
    st.stop_pending = 1;
  }
  st.run = 1;
  if (st.steps_left > 0) st.steps_left -= 1;
}

// Drainage structures (sfincs_discharges.f90:370-657), in order, after the
// boundary conditions of the step: each sets the discharge of its intake
// (qtsrc = -q) and outfall (+q), which the point-source kernel applies before
// continuity.  Levels are the FP32 state widened to FP64, as the reference
// evaluates them from its real*8 zs.
__device__ __forceinline__ void update_drainage(const ScnDev& S, const StepPlan& P) {
  const float dt = P.dt;
  const double t = P.t;
  for (int idrn = 0; idrn < S.ndrn; idrn++) {
    const DrnDev d = S.drn[idrn];
    const int jin = S.nsrc + 2 * idrn, jout = jin + 1;
    const double zin = (double)S.zs[d.cin], zout = (double)S.zs[d.cout];
    float qq = 0.0f;
    if (d.type == 1) {  // pump
      qq = d.p[0];
    } else if (d.type == 2 || d.type == 3) {  // culvert; check valve (intake to outfall only)
      if (zin > zout)
        qq = (float)((double)d.p[0] * sqrt(zin - zout));
      else
        qq = (float)((double)(-d.p[0]) * sqrt(zout - zin));
      if (d.type == 3) qq = fmaxf(qq, 0.0f);
    } else {  // gates: 4 opened while the intake level is in (zmin, zmax), 5 closed in [tclose, topen)
      const float wdt = d.p[0], zsill = d.p[1], mng = d.p[2], tcls = d.p[5];
      const float dzds = (float)((zout - zin) / (double)d.distance);
      float frac = S.drn_frac[idrn];
      const float hgate = (float)fmax(fmax(zin, zout) - (double)zsill, 0.0);
      const float dfrac = dt / tcls;
      const float qq0 = -S.qtsrc[jin] / (wdt * fmaxf(frac, 0.001f));
      int status = S.drn_status[idrn];
      if (d.type == 4) {
        if (status == 0) {
          if (zin > (double)d.p[3] && zin < (double)d.p[4]) status = 3;
        } else if (status == 1) {
          if (zin <= (double)d.p[3] || zin >= (double)d.p[4]) status = 2;
        }
      } else {
        if (status == 0) {
          if (t >= (double)d.p[4]) status = 3;
        } else if (status == 1) {
          if (t >= (double)d.p[3] && t < (double)d.p[4]) status = 2;
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
      S.drn_frac[idrn] = frac;
      S.drn_status[idrn] = status;
      // Bates et al. (2010) inertial flux; hgate**(7.0/3.0) as hgate**2 * cube_root(hgate)
      const float h73 = hgate * hgate * cube_root(hgate);
      qq = (qq0 - S.g * hgate * dzds * dt) / (1.0f + S.g * (mng * mng) * dt * fabsf(qq0) / h73);
      qq = qq * wdt * frac;
    }
    qq = 1.0f / (S.structure_relax / dt) * qq + (1.0f - (1.0f / (S.structure_relax / dt))) * -S.qtsrc[jin];
    // no more than the volume the giving cell holds
    if (S.subgrid) {
      if (qq > 0.0f)
        qq = (float)fmin((double)qq, fmax(S.zvol[d.cin], 0.0) / (double)dt);
      else
        qq = (float)fmax((double)qq, -fmax(S.zvol[d.cout], 0.0) / (double)dt);
    } else {
      const float ain = S.quadtree ? S.lv_area[S.qlev[d.cin]] : S.area;  // cell_area(z_flags_iref(nm))
      const float aout = S.quadtree ? S.lv_area[S.qlev[d.cout]] : S.area;
      if (qq > 0.0f)
        qq = (float)fmin((double)qq, fmax((zin - (double)S.zb[d.cin]) * (double)ain, 0.0) / (double)dt);
      else
        qq = (float)fmax((double)qq, -fmax((zout - (double)S.zb[d.cout]) * (double)aout, 0.0) / (double)dt);
    }
    S.qtsrc[jin] = -qq;
    S.qtsrc[jout] = qq;
  }
}

// --------------------------------------------------------------------------
// Boundary faces and Neumann cells.
// --------------------------------------------------------------------------
// Inputs of one boundary item that the kernel the step kernel waits for
// (continuity) does not write, read before the wait: the face record and the
// static tables, the running mean flux (written only by the step kernel), and
// the boundary-point levels of the time records the previous step used, which
// are the ones this step needs unless it crosses a record of the series.
struct BndPre {
  BndFace b;
  int2 nn;        // Neumann cell pair
  float2 zr;      // subgrid: z_zmin, z_zmax of the face
  float wx;       // subgrid: havg at z_zmax minus z_zmax, of the face
  float zbi;      // regular grids: bed level of the interior cell
  float um;       // running mean flux
  int itb0, itb1; // time records the point levels below belong to (0: none read)
  float z01[4];   // z0[i1], z1[i1], z0[i2], z1[i2]
};

__device__ __forceinline__ BndPre bnd_pre(const ScnDev& S, const StepState& st, int i) {
  BndPre r{};
  if (i < S.nkcuv2) {
    r.b = S.bfaces[i];
    const bool isv = r.b.info & 1;
    if (S.subgrid) {
      r.zr = isv ? S.sgz_v[r.b.face] : S.sgz_u[r.b.face];
      r.wx = (isv ? S.sgw_v[r.b.face] : S.sgw_u[r.b.face]).x;
    } else {
      r.zbi = S.zb[r.b.nmi];
    }
    r.um = S.uvmean[i];
    const int itb0 = st.itb0, itb1 = st.itb1;  // 0 before the first step
    if (!(r.b.info & (4 | 32)) && S.nbnd > 0 && itb0 >= 1 && itb0 <= S.ntbnd && itb1 >= 1 && itb1 <= S.ntbnd) {
      r.itb0 = itb0;
      r.itb1 = itb1;
      const int j1 = (r.b.info & 8) ? r.b.i1 : 0, j2 = (r.b.info & 8) ? r.b.i2 : 0;
      const float* z0 = S.zs_bnd + (size_t)(r.itb0 - 1) * S.nbnd;
      const float* z1 = S.zs_bnd + (size_t)(r.itb1 - 1) * S.nbnd;
      r.z01[0] = z0[j1];
      r.z01[1] = z1[j1];
      r.z01[2] = z0[j2];
      r.z01[3] = z1[j2];
    }
  } else if (i < S.nkcuv2 + S.nneu) {
    r.nn = S.neu[i - S.nkcuv2];
  }
  return r;
}

// Inputs of one boundary item that the previous kernel writes, read right
// after the wait for it, before any of this thread's stores (a later item's
// loads could otherwise not be issued ahead of an earlier item's stores).
struct BndDyn {
  float zsnmi;     // level of the interior cell (Neumann: of the source cell)
  bool vol_dry;    // subgrid: the interior cell's volume is not positive
  float zsmax;     // running maximum of the boundary cell
};

__device__ __forceinline__ BndDyn bnd_dyn(const ScnDev& S, int i, const BndPre& pre) {
  BndDyn d{};
  if (i < S.nkcuv2) {
    d.zsnmi = S.zs[pre.b.nmi];
    d.vol_dry = S.subgrid && S.zvol[pre.b.nmi] <= 0.0;
    if (S.store_zsmax) d.zsmax = S.zsmax[pre.b.nmb];
  } else if (i < S.nkcuv2 + S.nneu) {
    d.zsnmi = S.zs[pre.nn.y];
  }
  return d;
}

// One water-level boundary face (i < nkcuv2) or Neumann cell: returns its FP64
// inflow volume this step.
__device__ __forceinline__ double boundary_item(const ScnDev& S, const StepPlan& P, int i, BndPre pre,
                                                const BndDyn& dyn) {
  double inflow = 0.0;
  if (i < S.nkcuv2) {
    const BndFace& b = pre.b;
    const bool isv = b.info & 1;
    const float sgn = (b.info & 2) ? 1.0f : -1.0f;
    const int p = P.parity;
    const float dt = P.dt;
    const double t = P.t;
    const float zsnmi = dyn.zsnmi;
    const bool vol_dry = dyn.vol_dry;
    // level of the boundary cell (sfincs_boundaries.f90:728-756, 800-876)
    float zsnmb, zs0nmb;
    if (b.info & 4) {
      zsnmb = zs0nmb = b.zfix;
    } else if (b.info & 32) {  // downstream river: internal level plus the slope drop, not below the floor (:878-902)
      zsnmb = zs0nmb = (float)fmax((double)S.zs[b.zsi] + (double)b.zfix, (double)b.floor);
    } else {
      if (S.nbnd > 0 && (pre.itb0 != P.itb0 || pre.itb1 != P.itb1)) {  // not read ahead, or another time record
        const int j1 = (b.info & 8) ? b.i1 : 0, j2 = (b.info & 8) ? b.i2 : 0;
        const float* z0 = S.zs_bnd + (size_t)(P.itb0 - 1) * S.nbnd;
        const float* z1 = S.zs_bnd + (size_t)(P.itb1 - 1) * S.nbnd;
        pre.z01[0] = z0[j1];
        pre.z01[1] = z1[j1];
        pre.z01[2] = z0[j2];
        pre.z01[3] = z1[j2];
      }
      // levels at the two boundary points (:728-756), then the face's weighted level
      float zp1 = pre.z01[0] + (pre.z01[1] - pre.z01[0]) * P.tbfac;
      float zp2 = pre.z01[2] + (pre.z01[3] - pre.z01[2]) * P.tbfac;
      if (S.ntide > 0) {  // astronomic constituents (:736-744)
        zp1 = tide_level(S, (b.info & 8) ? b.i1 : 0, t, zp1);
        if (b.info & 8) zp2 = tide_level(S, b.i2, t, zp2);
      }
      double zst;
      if (b.info & 8)
        zst = (double)(zp1 * b.fac + zp2 * (1.0f - b.fac));
      else
        zst = (double)zp1;
      if (S.patmos && S.pavbnd > 1.0f)  // barometric correction with the boundary cell's pressure (:820-826)
        zst = zst + (double)((S.pavbnd - cell_patm(S, b.nmb, meteo_weights(S, t, P.mt0, P.mt1))) / (S.rhow * 9.81f));
      float zb0;
      if (t < (double)(S.tspinup - 1.0e-3f)) {
        const float smfac = (float)(1.0 - (t - (double)S.t0) / (double)(S.tspinup - S.t0));
        zb0 = S.zini * smfac + (float)zst * (1.0f - smfac);
      } else {
        zb0 = (float)zst;
      }
      zsnmb = zs0nmb = fmaxf(zb0, b.floor);
    }
    const float zsb_v = zsnmb;
    // weakly reflective flux (sfincs_boundaries.f90:968-1093)
    float hnmb;
    if (S.subgrid) {
      const float2 zr = pre.zr;
      const float zsuv = fmaxf(zsnmb, zsnmi);
      float depthuv;
      if (zsuv >= zr.y - 1.0e-4f) {
        depthuv = pre.wx + zsuv;
      } else if (zsuv > zr.x) {
        const float dzuv = (zr.y - zr.x) / (float)(S.nlev - 1);
        const int iuv = lev_index((zsuv - zr.x) / dzuv, S.nlev);
        const float facint = (zsuv - (zr.x + (float)(iuv - 1) * dzuv)) / dzuv;
        const UvRec r = (isv ? S.rec_v : S.rec_u)[(int64_t)(iuv - 1) * S.nalloc + b.face];
        depthuv = r.havg + r.dhavg * facint;
      } else {
        depthuv = 0.0f;
      }
      hnmb = fmaxf(depthuv, S.huthresh);
    } else {
      hnmb = fmaxf(0.5f * (zsnmb + zsnmi) - b.zbuv, S.huthresh);
    }
    zsnmb = fmaxf(zsnmb, b.floor);
    zs0nmb = fmaxf(zs0nmb, b.floor);
    float qq = 0.0f, uu = 0.0f;
    float um = pre.um;
    if (hnmb < S.huthresh + 1.0e-6f || (b.info & 16)) {  // bit 4: a weir sits on this face (kcuv 3)
      um = 0.0f;
    } else {
      const float sq = sqrtf(S.g / hnmb);
      const float ui = sq * (zsnmb - zs0nmb);
      const float ubv = sgn * (2.0f * ui - sq * (zsnmi - zs0nmb));
      qq = ubv * hnmb + um;
      if (S.subgrid) {
        if (vol_dry) qq = sgn > 0.0f ? fmaxf(qq, 0.0f) : fminf(qq, 0.0f);
        if (zsnmb - b.floor < S.huthresh) qq = sgn > 0.0f ? fminf(qq, 0.0f) : fmaxf(qq, 0.0f);
      } else {
        if (zsnmi - pre.zbi <= S.huthresh) qq = sgn > 0.0f ? fmaxf(qq, 0.0f) : fminf(qq, 0.0f);
        if (zsnmb - b.floor < S.huthresh) qq = sgn > 0.0f ? fminf(qq, 0.0f) : fmaxf(qq, 0.0f);
      }
      uu = fmaxf(fminf(qq / hnmb, 4.0f), -4.0f);
    }
    // boundary faces are not momentum faces: write both ping-pong buffers
    float* const* Q = isv ? S.qv : S.qu;
    float* const* U = isv ? S.vv : S.uu;
    Q[p][b.face] = qq;
    Q[p ^ 1][b.face] = qq;
    U[p][b.face] = uu;
    U[p ^ 1][b.face] = uu;
    if (S.btfilter >= -1.0e-6f) {
      const float factime = fminf(dt / S.btfilter, 1.0f);
      const float facrel = 1.0f - fminf(dt / S.btrelax, 1.0f);
      S.uvmean[i] = factime * qq + facrel * (1.0f - factime) * um;
    } else {
      S.uvmean[i] = 0.0f;
    }
    S.zs[b.nmb] = zsb_v;
    if (S.store_zsmax) {  // sfincs_boundaries.f90:1101-1113
      if (S.store_tzsmax && zsb_v > dyn.zsmax) S.tzsmax[b.nmb] = (float)P.t;
      S.zsmax[b.nmb] = fmaxf(dyn.zsmax, zsb_v);
    }
    inflow = (double)sgn * (double)qq * (double)b.len * (double)dt;
  } else if (i < S.nkcuv2 + S.nneu) {
    S.zs[pre.nn.x] = dyn.zsnmi;  // Neumann: zs(nmb) = zs(nmi) (sfincs_boundaries.f90:903-914)
  }
  return inflow;
}

// FP64 volume-balance accumulator of the boundary inflow: block sum, one
// atomic.  Every thread of the block passes its barrier.
__device__ __forceinline__ void add_inflow(StepState& st, double inflow) {
  __shared__ double s_red[32];
  inflow = warp_sum(inflow);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = inflow;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += s_red[w];
    if (tot != 0.0) atomicAdd(&st.bflux_vol, tot);
  }
}

// Step control and all boundary faces of one scenario in one CTA (ONE: the
// single scenario's parameters by value).  This kernel's time is its chain of
// dependent memory accesses, so the chain is kept short:
// - the inputs of each thread's first two boundary items that the previous
//   kernel does not write are read before the kernel waits for it, the others
//   right after the wait, together with the step state;
// - every thread derives the step plan from the same loads of the step state;
// - the last thread, which has the fewest boundary items, then reads the
//   forcing time series while the others finish theirs;
// - thread 0 commits the plan after the barrier of the inflow sum, when no
//   thread reads the step state any more, and then updates the drainage
//   structures, which read the boundary cells' new levels.
template <bool ONE>
__global__ void __launch_bounds__(1024) k_step_bnd(const ScnDev* __restrict__ scns, const __grid_constant__ ScnDev one) {
  const ScnDev& S = ONE ? one : scns[blockIdx.x];
  StepState& st = *S.st;
  const int nitems = S.nkcuv2 + S.nneu;
  const int i0 = threadIdx.x, i1 = threadIdx.x + blockDim.x;
  const BndPre pre0 = bnd_pre(S, st, i0);
  const BndPre pre1 = bnd_pre(S, st, i1);
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const BndDyn dyn0 = bnd_dyn(S, i0, pre0);
  const BndDyn dyn1 = bnd_dyn(S, i1, pre1);
  const StepPlan P = plan_step(S, st);
  double inflow = 0.0;
  if (P.go) {
    if (i0 < nitems) inflow += boundary_item(S, P, i0, pre0, dyn0);
    if (i1 < nitems) inflow += boundary_item(S, P, i1, pre1, dyn1);
    for (int i = i1 + (int)blockDim.x; i < nitems; i += blockDim.x) {
      const BndPre pre = bnd_pre(S, st, i);
      inflow += boundary_item(S, P, i, pre, bnd_dyn(S, i, pre));
    }
    if (threadIdx.x == blockDim.x - 1) step_forcing(S, st, P);
  }
  add_inflow(st, inflow);  // also orders the boundary cells' levels before the drainage reads them
  if (threadIdx.x == 0) {
    commit_step(S, st, P);
    if (P.go && S.ndrn > 0) update_drainage(S, P);
    // Green-Ampt reads GA_head(np) * GA_sigma(np) for every cell
    // (sfincs_infiltration.f90:858): the last cell's values before this step's update
    if (P.go && S.inftype == 4) st.ga_hs = S.inf_par[4][S.inf_last] * S.inf_st[0][S.inf_last];
  }
}

// --------------------------------------------------------------------------
// Gridded meteo: the two fields of an update window on the cells.
// --------------------------------------------------------------------------
// The records around one end of the window (update_amuv_data and its
// pressure / rain twins, sfincs_meteo.f90:823-845, 998-1020, 1128-1155).
struct MeteoRec {
  int i0, i1;  // 0-based records
  float twfac;
};
__device__ __forceinline__ MeteoRec meteo_rec(const MeteoGrid& g, float meteo_t, bool block) {
  meteo_t = fmaxf(meteo_t, g.times[0]);
  meteo_t = fminf(meteo_t, g.times[g.nt - 1]);
  int itw0 = 1;
  for (int it = 1; it <= g.nt; it++)
    if (g.times[it - 1] <= meteo_t) itw0 = it;
  const int itw1 = min(itw0 + 1, g.nt);
  meteo_t = fminf(meteo_t, g.times[itw1 - 1]);
  MeteoRec r;
  r.i0 = itw0 - 1;
  r.i1 = itw1 - 1;
  r.twfac = block ? 0.0f : (meteo_t - g.times[itw0 - 1]) / fmaxf(g.times[itw1 - 1] - g.times[itw0 - 1], 1.0e-6f);
  return r;
}

// Bilinear interpolation of quantity v (records blended by r) at (x, y), in
// the reference's index arithmetic (:851-898); false outside the grid (the
// reference treats the first row band and the edges as outside too).
__device__ __forceinline__ bool meteo_at(const MeteoGrid& g, const float* v, const float* v2, const MeteoRec& r,
                                         float x, float y, float& out, float& out2) {
  const float yul = g.y_ll + (float)(g.nrows - 1) * g.dy + 0.5f * g.dy;
  const float xll = g.x_ll + 0.5f * g.dx;
  const int iy = (int)((yul - y) / g.dy) + 1;
  const float dj1 = (yul - (float)(iy - 1) * g.dy - y) / g.dy;
  const int ix = (int)((x - xll) / g.dx) + 1;
  const float di1 = (x - (xll + (float)(ix - 1) * g.dx)) / g.dx;
  if (iy <= 1 || iy >= g.nrows || ix <= 0 || ix >= g.ncols) return false;
  const int ind1[4] = {iy, iy, iy + 1, iy + 1}, ind2[4] = {ix, ix + 1, ix + 1, ix};
  const float f[4] = {(1.0f - di1) * (1.0f - dj1), di1 * (1.0f - dj1), di1 * dj1, (1.0f - di1) * dj1};
  const size_t rec = (size_t)g.nrows * g.ncols;
  float a = 0.0f, b = 0.0f;
  for (int ip = 0; ip < 4; ip++) {
    const size_t o = (size_t)(ind1[ip] - 1) * g.ncols + (ind2[ip] - 1);
    a = a + f[ip] * (v[r.i0 * rec + o] * (1.0f - r.twfac) + v[r.i1 * rec + o] * r.twfac);
    if (v2) b = b + f[ip] * (v2[r.i0 * rec + o] * (1.0f - r.twfac) + v2[r.i1 * rec + o] * r.twfac);
  }
  out = a;
  out2 = b;
  return true;
}

// The records around one end of the window in a spiderweb and its eye
// (update_spiderweb_data, sfincs_meteo.f90:485-531): before the first record
// and after the last the nearest record, faded in / out over 6 h.
struct SpwRec {
  int i0, i1;  // 0-based records
  float twfac, spin, xe, ye;
};
__device__ __forceinline__ SpwRec spw_rec(const SpwGrid& g, float meteo_t) {
  SpwRec r;
  int itw0 = 1, itw1 = 1;
  r.twfac = 1.0f;
  r.spin = 1.0f;
  if (meteo_t < g.times[0]) {
    r.spin = fmaxf(1.0f - (g.times[0] - meteo_t) / 21600.0f, 0.0f);
  } else if (meteo_t > g.times[g.nt - 1]) {
    itw0 = itw1 = g.nt;
    r.spin = fmaxf(1.0f - (meteo_t - g.times[g.nt - 1]) / 21600.0f, 0.0f);
  } else {
    for (int it = 1; it <= g.nt; it++)
      if (g.times[it - 1] <= meteo_t) itw0 = it;
    itw1 = min(itw0 + 1, g.nt);
    r.twfac = (meteo_t - g.times[itw0 - 1]) / fmaxf(g.times[itw1 - 1] - g.times[itw0 - 1], 1.0e-6f);
  }
  r.i0 = itw0 - 1;
  r.i1 = itw1 - 1;
  r.xe = g.xe[r.i0] * (1.0f - r.twfac) + g.xe[r.i1] * r.twfac;
  r.ye = g.ye[r.i0] * (1.0f - r.twfac) + g.ye[r.i1] * r.twfac;
  return r;
}

// Merges the spiderweb into one cell's window values at one end (the
// per-cell loop of update_spiderweb_data, sfincs_meteo.f90:589-790): the
// polar bilinear weights around the eye, the drag of the interpolated wind,
// and the blend with the background fields towards the web's rim.
__device__ __forceinline__ void spw_merge(const ScnDev& S, const SpwRec& r, float x, float y, float& tu, float& tv,
                                          float& p, float& pr) {
  const SpwGrid& g = S.spw;
  const float dxe = x - r.xe, dye = y - r.ye;
  const float dst = sqrtf(dxe * dxe + dye * dye);
  if (dst > g.radius) return;  // outside the web
  const int idst = max((int)(dst / g.drad), 1);
  if (idst + 1 > g.nrows) return;
  const float dj1 = fmaxf((dst - g.drad * (float)idst) / g.drad, 0.0f);
  float phi = 0.5f * S.pi - atan2_ieee(dye, dxe);  // clockwise from north
  if (phi < 0.0f) phi = phi + 2.0f * S.pi;          // modulo 2 pi (phi > -pi here)
  const int iphi = min((int)(phi / g.dphi) + 1, g.ncols);
  const int ind1[4] = {idst, idst, idst + 1, idst + 1};
  int ind2[4] = {iphi, iphi + 1, iphi + 1, iphi};
  if (ind2[1] > g.ncols) ind2[1] = 1;
  if (ind2[2] > g.ncols) ind2[2] = 1;
  const float di1 = (phi - g.dphi * (float)(iphi - 1)) / g.dphi;
  const float f[4] = {(1.0f - di1) * (1.0f - dj1), di1 * (1.0f - dj1), di1 * dj1, (1.0f - di1) * dj1};
  const size_t rec = (size_t)g.nrows * g.ncols;
  const float a = 1.0f - r.twfac, b = r.twfac;
  float wup = 0.0f, wvp = 0.0f, pcp = 0.0f, prp = 0.0f;
  for (int ip = 0; ip < 4; ip++) {
    const size_t o = (size_t)(ind1[ip] - 1) * g.ncols + (ind2[ip] - 1);
    const size_t o0 = r.i0 * rec + o, o1 = r.i1 * rec + o;
    wup = wup + f[ip] * (g.wu[o0] * a + g.wu[o1] * b);
    wvp = wvp + f[ip] * (g.wv[o0] * a + g.wv[o1] * b);
    if (S.patmos) pcp = pcp + f[ip] * (g.pabs[o0] * a + g.pabs[o1] * b);
    if (g.precip) prp = prp + f[ip] * (g.prcp[o0] * a + g.prcp[o1] * b);
  }
  const float vmag = sqrtf(wup * wup + wvp * wvp);
  const int icd = min(max((int)(vmag * 10.0f) + 1, 1), 1000);
  const float cd = S.cdval[icd - 1];
  float merge = 1.0f;
  if (dst > g.merge_frac * g.radius)
    merge = (1.0f / (1.0f - fminf(g.merge_frac, 0.999f))) * (g.radius - dst) / g.radius;
  merge = merge * r.spin;
  tu = (1.0f - merge) * tu + merge * vmag * (S.cosrot * wup + S.sinrot * wvp) * S.rhoa * cd / S.rhow;
  tv = (1.0f - merge) * tv + merge * vmag * (-S.sinrot * wup + S.cosrot * wvp) * S.rhoa * cd / S.rhow;
  if (S.patmos) p = (1.0f - merge) * p + merge * pcp;
  if (g.precip) pr = (1.0f - merge) * pr + merge * prp / (float)(1000 * 3600);
}

// Runs before the step kernel: when the step about to run opens a new window
// (the same decision the step kernel commits), every cell gets the window's
// wind stress, pressure and rain at both ends (update_meteo_fields,
// sfincs_meteo.f90:1561-1624: the equidistant grids, then the spiderweb
// merged over them); otherwise every CTA returns at once.
__global__ void __launch_bounds__(256) k_meteo_window(const ScnDev* __restrict__ scns) {
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const ScnDev& S = scns[blockIdx.y];
  if (!S.meteo3d) return;
  const StepState& st = *S.st;
  const StepPlan P = plan_step(S, st);
  if (!P.meteo_upd) return;
  __shared__ MeteoRec recs[3][2];
  __shared__ SpwRec srecs[2];
  if (threadIdx.x < 6) {
    const int kind = threadIdx.x >> 1, itw = threadIdx.x & 1;
    const MeteoGrid& g = S.mg[kind];
    if (g.nt > 0) recs[kind][itw] = meteo_rec(g, itw == 0 ? P.mt0 : P.mt1, kind == 2 && S.ampr_block);
  } else if (threadIdx.x < 8 && S.spw.nt > 0) {
    srecs[threadIdx.x - 6] = spw_rec(S.spw, threadIdx.x == 6 ? P.mt0 : P.mt1);
  }
  __syncthreads();
  const float cosrot = S.cosrot, sinrot = S.sinrot;
  const bool wf = S.wind_field, pf = S.patmos, rf = S.prcp_field;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.nmeteo; i += gridDim.x * blockDim.x) {
    const int64_t c = S.cmp ? (int64_t)S.cmp[i] : (int64_t)i;
    const float x = S.xz[i], y = S.yz[i];
    for (int itw = 0; itw < 2; itw++) {
      float tu = 0.0f, tv = 0.0f, p = S.gapres, pr = 0.0f;
      if (S.mg[0].nt > 0) {  // wind stress (:862-936), outside the grid 0
        float wup, wvp;
        if (meteo_at(S.mg[0], S.mg[0].v0, S.mg[0].v1, recs[0][itw], x, y, wup, wvp)) {
          const float vmag = sqrtf(wup * wup + wvp * wvp);
          const int icd = min(max((int)(vmag * 10.0f) + 1, 1), 1000);
          const float cd = S.cdval[icd - 1];
          tu = vmag * (cosrot * wup + sinrot * wvp) * S.rhoa * cd / S.rhow;
          tv = vmag * (-sinrot * wup + cosrot * wvp) * S.rhoa * cd / S.rhow;
        }
      }
      if (S.mg[1].nt > 0 && pf) {  // pressure (:1035-1080), outside the grid gapres
        float v, unused;
        if (meteo_at(S.mg[1], S.mg[1].v0, nullptr, recs[1][itw], x, y, v, unused)) p = v;
      }
      if (S.mg[2].nt > 0) {  // rain in mm/h to m/s (:1160-1232), outside the grid 0
        float v, unused;
        if (meteo_at(S.mg[2], S.mg[2].v0, nullptr, recs[2][itw], x, y, v, unused)) pr = v / (float)(1000 * 3600);
      }
      if (S.spw.nt > 0) spw_merge(S, srecs[itw], x, y, tu, tv, p, pr);
      if (wf) {
        (itw == 0 ? S.tauwu0 : S.tauwu1)[c] = tu;
        (itw == 0 ? S.tauwv0 : S.tauwv1)[c] = tv;
      }
      if (pf) (itw == 0 ? S.patm0 : S.patm1)[c] = p;
      if (rf) (itw == 0 ? S.prcp0 : S.prcp1)[c] = pr;
    }
  }
}

void launch_meteo_window(const ScnDev* d_scns, int nscn, int max_cells, cudaStream_t s) {
  const int blocks = max(1, min((max_cells + 255) / 256, 1184));
  launch_pdl(k_meteo_window, dim3(blocks, nscn), dim3(256), 0, s, d_scns);
}

// --------------------------------------------------------------------------
// k_momentum: one thread per uv face.
// --------------------------------------------------------------------------
template <bool SG, int DIR>
__device__ __forceinline__ float momentum_face(const ScnDev& S, const StepVals& sv, int64_t c) {
  const int p = sv.parity;
  const int64_t ld = S.ld;
  const int64_t du = DIR == 0 ? ld : 1;  // to the cell across the face (nmu)
  const int64_t dq = DIR == 0 ? 1 : ld;  // transverse direction
  constexpr uint16_t ACT = DIR == 0 ? F_UACT : F_VACT;
  constexpr uint16_t ADV = DIR == 0 ? F_UADV : F_VADV;
  constexpr uint16_t TH = DIR == 0 ? F_UTH : F_VTH;
  constexpr uint16_t NDM = DIR == 0 ? F_CDN : F_CLF;
  constexpr uint16_t NUM = DIR == 0 ? F_CUP : F_CRT;
  // ---- wave 1: independent loads (speculative: every address is inside the dense arrays)
  const uint16_t f = S.flags[c];
  const float zs_nm = S.zs[c];
  const float zs_nmu = S.zs[c + du];
  uint8_t* __restrict__ kfp = S.kf[DIR];
  const uint8_t kf = kfp[c];
  float zmin, zmax;
  if (SG) {
    const float2 zr = (DIR == 0 ? S.sgz_u : S.sgz_v)[c];
    zmin = zr.x;
    zmax = zr.y;
  } else {
    zmin = (DIR == 0 ? S.zbmx_u : S.zbmx_v)[c];
    zmax = 0.0f;
  }
  if (!(f & ACT)) return FLT_MAX;
  float* __restrict__ Qn = (DIR == 0 ? S.qu : S.qv)[p ^ 1];
  float* __restrict__ Un = (DIR == 0 ? S.uu : S.vv)[p ^ 1];
  const float zsu = fmaxf(zs_nm, zs_nmu);
  const bool wet = SG ? (zsu > zmin + S.huthresh) : (zsu > zmin);
  if (!wet) {  // sfincs_momentum.f90:743-748
    if (kf & KF_WET2) {  // the buffer being written may still hold the value of two steps ago
      Qn[c] = 0.0f;
      Un[c] = 0.0f;
    }
    const uint8_t kfn = (uint8_t)((kf & (KF_WET | KF_STALE)) ? KF_WET2 : 0);
    if (kfn != kf) kfp[c] = kfn;
    return FLT_MAX;
  }
  // ---- wave 2: neighbours, table record, limiter inputs (all independent)
  const float* __restrict__ Q = (DIR == 0 ? S.qu : S.qv)[p];
  const float* __restrict__ T = (DIR == 0 ? S.qv : S.qu)[p];
  const float* __restrict__ U = (DIR == 0 ? S.uu : S.vv)[p];
  const float* __restrict__ V = (DIR == 0 ? S.vv : S.uu)[p];
  const float qx_nm = Q[c], qx_nmd = Q[c - du], qx_nmu = Q[c + du];
  const float qy_nm = T[c], qy_nmu = T[c + du], qy_ndm = T[c - dq], qy_ndmu = T[c + du - dq];
  const float uu_nm = U[c], uu_nmd = U[c - du], uu_nmu = U[c + du];
  const float uu_ndm = (f & NDM) ? U[c - dq] : uu_nm;
  const float uu_num = (f & NUM) ? U[c + dq] : uu_nm;
  const float v0 = V[c - dq], v1 = V[c + du - dq], v2 = V[c], v3 = V[c + du];
  float hu, gnavg2, phi = 1.0f;
  bool dry_nm, dry_nmu;
  float zd_nm = 0.0f, zd_nmu = 0.0f;
  if (SG) {
    dry_nm = S.vneg[c] != 0;
    dry_nmu = S.vneg[c + du] != 0;
    if (S.wiggle) {
      zd_nm = S.zsderv[c];
      zd_nmu = S.zsderv[c + du];
    }
    if (zsu > zmax) {  // sfincs_momentum.f90:347-366
      const float4 w = (DIR == 0 ? S.sgw_u : S.sgw_v)[c];
      hu = w.x + zsu;
      gnavg2 = sg_gnavg2_full(w.z, w.y, w.w, zsu - zmax);
    } else {  // sfincs_momentum.f90:372-378
      const SgLevel lv = sg_level(zsu, zmin, zmax, S.nlev);
      const UvRec r = (DIR == 0 ? S.rec_u : S.rec_v)[(int64_t)(lv.iuv - 1) * S.nalloc + c];
      hu = fmaf(r.dhavg, lv.facint, r.havg);
      gnavg2 = fmaf(r.dnrep, lv.facint, r.nrep);
      phi = fmaf(r.dpwet, lv.facint, r.pwet);
    }
  } else {  // sfincs_momentum.f90:384-385
    dry_nm = zs_nm < S.zb[c];
    dry_nmu = zs_nmu < S.zb[c + du];
    hu = fmaxf(zsu - zmin, S.huthresh);
    gnavg2 = (DIR == 0 ? S.gn2_u : S.gn2_v)[c];
  }
  FaceGeo geo;
  if (S.geo) {  // geographic: the cell's width across x, in metres (sfincs_momentum.f90:205-217)
    const float dxm_inv = S.geo_dxminv[c];
    geo.dxuvinv = DIR == 0 ? dxm_inv : S.dyinv;
    geo.dyuvinv = DIR == 0 ? S.dyinv : dxm_inv;
    geo.dxuv2inv = DIR == 0 ? dxm_inv * dxm_inv : S.dy2inv;
    geo.dyuv2inv = DIR == 0 ? S.dy2inv : dxm_inv * dxm_inv;
    geo.fcorio = S.geo_fcor ? S.geo_fcor[c] : 0.0f;
  } else {
    geo.dxuvinv = DIR == 0 ? S.dxinv : S.dyinv;
    geo.dyuvinv = DIR == 0 ? S.dyinv : S.dxinv;
    geo.dxuv2inv = DIR == 0 ? S.dx2inv : S.dy2inv;
    geo.dyuv2inv = DIR == 0 ? S.dy2inv : S.dx2inv;
    geo.fcorio = S.fcorio;
  }
  geo.nuvisc = S.nuvisc;
  FaceV a;
  a.qx_nm = qx_nm;
  a.qx_nmd = qx_nmd;
  a.qx_nmu = qx_nmu;
  a.qy_nm = qy_nm;
  a.qy_nmu = qy_nmu;
  a.qy_ndm = qy_ndm;
  a.qy_ndmu = qy_ndmu;
  a.uu_nm = uu_nm;
  a.uu_nmd = uu_nmd;
  a.uu_nmu = uu_nmu;
  a.uu_ndm = uu_ndm;
  a.uu_num = uu_num;
  a.vu = (v0 + v1 + v2 + v3) / 4.0f;
  float q, uv, tauw, dpatm;
  face_meteo(S, sv, DIR, c, c + du, tauw, dpatm);
  const float ghu = face_flux_geo<SG>(S, sv, DIR, (f & ADV) != 0, (f & TH) != 0, geo, kf, zs_nm, zs_nmu, hu, gnavg2,
                                      phi, a, dry_nm, dry_nmu, zd_nm, zd_nmu, tauw, dpatm, q, uv);
  const float den = fmaxf(sqrtf(ghu), fabsf(uv)) * geo.dxuvinv;
  Qn[c] = q;
  Un[c] = uv;
  const uint8_t kfn = (uint8_t)(KF_WET | ((kf & (KF_WET | KF_STALE)) ? KF_WET2 : 0));
  if (kfn != kf) kfp[c] = kfn;
  return 1.0f / den;  // sfincs_momentum.f90:731
}

template <bool SG, int MINB>
__global__ void __launch_bounds__(512, MINB) k_momentum(const ScnDev* __restrict__ scns, const Tile* __restrict__ tiles) {
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const Tile tl = tiles[blockIdx.x];
  const ScnDev& S = scns[tl.scn];
  const StepState& st = *S.st;
  if (!st.run) return;
  const StepVals sv = step_vals(st);
  const int n = tl.n0 + threadIdx.x;
  const int m = tl.m0 + threadIdx.y;
  float mdt = FLT_MAX;
  if (n <= S.nmax && m <= S.mmax) {
    const int64_t c = off(S, n, m);
    mdt = threadIdx.z == 0 ? momentum_face<SG, 0>(S, sv, c) : momentum_face<SG, 1>(S, sv, c);
  }
  // CTA min of the CFL time step, then one atomicMin per CTA (float bits of a positive value)
  __shared__ float s_min[16];
  mdt = warp_min(mdt);
  const int lane = threadIdx.x;
  const int warp = threadIdx.y + threadIdx.z * blockDim.y;
  if (lane == 0) s_min[warp] = mdt;
  __syncthreads();
  if (warp == 0) {
    float v = lane < (int)(blockDim.y * blockDim.z) ? s_min[lane] : FLT_MAX;
    v = warp_min(v);
    if (lane == 0 && v < FLT_MAX) atomicMin(&S.st->min_dt_bits, __float_as_uint(v));
  }
}

// --------------------------------------------------------------------------
// Point sources, applied in the reference's sequential order before the cell loop.
// --------------------------------------------------------------------------
__global__ void k_sources(const ScnDev* __restrict__ scns) {
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const ScnDev& S = scns[blockIdx.x];
  StepState& st = *S.st;
  if (!st.run || S.nsrc + S.ndrn == 0 || threadIdx.x != 0) return;
  const float dt = st.dt;
  double vol = 0.0;
  for (int is = 0; is < S.nsrc + 2 * S.ndrn; is++) {
    const int c = S.src_cell[is];
    if (S.subgrid) {
      if (S.zvol[c] >= 0.0) {
        S.zvol[c] = S.zvol[c] + (double)(S.qtsrc[is] * dt);
        vol += (double)(S.qtsrc[is] * dt);
      }
    } else {
      const float area = S.geo ? S.geo_area[c] : S.quadtree ? S.lv_area[S.qlev[c]] : S.area;  // cell_area(_m2)
      const float before = S.zs[c];
      const float z = fmaxf(S.zs[c] + S.qtsrc[is] * dt / area, S.zb[c]);
      S.zs[c] = z;
      vol += ((double)z - (double)before) * (double)area;
    }
  }
  st.src_vol += vol;
}

// --------------------------------------------------------------------------
// Weirs: fluxes over structure faces after the momentum faces
// (sfincs_structures.f90:592-697), one CTA per scenario.  The flux goes into
// the buffers this step's momentum wrote, which continuity reads.
// --------------------------------------------------------------------------
__global__ void k_structures(const ScnDev* __restrict__ scns) {
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const ScnDev& S = scns[blockIdx.x];
  const StepState& st = *S.st;
  if (!st.run) return;
  const int p1 = st.parity ^ 1;
  for (int i = threadIdx.x; i < S.nstruc; i += blockDim.x) {
    const StrucFace w = S.struc[i];
    float* Q = w.dir == 0 ? S.qu[p1] : S.qv[p1];
    float* U = w.dir == 0 ? S.uu[p1] : S.vv[p1];
    const float zsnm = S.zs[w.nm], zsnmu = S.zs[w.nmu];
    float q = 0.0f;
    if (!(zsnm < w.height && zsnmu < w.height)) {
      // broad-crested weir (type 1): submerged or free flow
      const float cweir = 1.7049f, mlim = 0.0f;
      float h1, h2, idir;
      if (zsnm > zsnmu) {
        idir = 1.0f;
        h1 = zsnm - w.height;
        h2 = zsnmu - w.height;
      } else {
        idir = -1.0f;
        h1 = zsnmu - w.height;
        h2 = zsnm - w.height;
      }
      float qstruc;
      if (h2 > 2.0f / 3.0f * h1)
        qstruc = w.cd * h2 * sqrtf(2.0f * 9.81f * (h1 - h2) / (1.0f - mlim));
      else  // h1**1.5 as h1 * sqrt(h1): two correctly rounded operations, within 1.5 ulp of the power
        qstruc = w.cd * cweir * (h1 * sqrtf(h1));
      qstruc = qstruc * w.len;
      q = qstruc * idir;
    }
    Q[w.face] = q;
    U[w.face] = 0.0f;
  }
}

// --------------------------------------------------------------------------
// Continuity: one thread per cell.
// --------------------------------------------------------------------------
template <bool SG>
__global__ void __launch_bounds__(256) k_continuity(const ScnDev* __restrict__ scns, const Tile* __restrict__ tiles) {
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const Tile tl = tiles[blockIdx.x];
  const ScnDev& S = scns[tl.scn];
  const StepState& st = *S.st;
  if (!st.run) return;
  const int n = tl.n0 + threadIdx.x;
  const int m = tl.m0 + threadIdx.y;
  if (n > S.nmax || m > S.mmax) return;
  const int64_t c = off(S, n, m);
  const int64_t ld = S.ld;
  const int p1 = st.parity ^ 1;  // buffers written by this step's momentum
  // ---- wave 1: everything whose address is known (speculative inside the dense arrays)
  const uint16_t f = S.flags[c];
  const float* __restrict__ qu = S.qu[p1];
  const float* __restrict__ qv = S.qv[p1];
  const float q_md = qu[c - ld], q_mu = qu[c], q_nd = qv[c - 1], q_nu = qv[c];
  const float zs_old = S.zs[c];
  const float zm = S.zsmax[c];
  const float qx = S.use_qext ? S.qext[c] : 0.0f;
  const float qi = S.infiltration ? S.qinf[c] : 0.0f;
  double v_old = 0.0;
  float zs00 = 0.0f, volmax = 0.0f;
  uint8_t vn_old = 0;
  float zbc = 0.0f;
  if (SG) {
    v_old = S.zvol[c];
    volmax = S.zz_volmax[c];
    vn_old = S.vneg[c];
    if (S.wiggle) zs00 = S.zs0[c];
  } else if (S.infiltration) {
    zbc = S.zb[c];
  }
  if (!(f & F_ACT)) return;
  const float dt = st.dt;
  float zsn = zs_old;
  const float area = S.geo ? S.geo_area[c] : S.area;  // cell_area_m2 on geographic grids (:458-470)
  // infiltration with state (or cumulative rain) for every active cell, from the start-of-step state
  const bool inf_cell = S.precip && (S.inftype >= 2 || S.store_cumprcp);
  float qinf_cell = 0.0f;
  // rain of the cell: uniform from a time series, or from the gridded field
  float prc = st.ptmp, netr = st.ptmp;
  if (S.prcp_field)
    prc = cell_rain(S, c, meteo_weights(S, st.t, st.meteo_t0, st.meteo_t1), SG ? v_old <= 0.0 : zs_old <= S.zb[c],
                    netr);
  if (inf_cell) {
    if (SG) {
      qinf_cell = cell_infiltration(S, c, prc, dt, v_old <= 0.0, (float)(v_old / (double)area), st.ga_hs);
    } else {
      const float zb0 = S.zb[c];
      qinf_cell = cell_infiltration(S, c, prc, dt, zs_old <= zb0, (float)((double)zs_old - (double)zb0), st.ga_hs);
    }
  }
  if (S.qinfmap) store_qinfmap(S, c, inf_cell, qinf_cell, SG ? v_old > 0.0 : !(zs_old <= S.zb[c]));
  if (f & F_KCS1) {
    if (SG) {  // sfincs_continuity.f90:341-577
      // geographic: the face lengths are dyrm and the cell's width dxm (:350-361)
      float dvol = S.geo ? ((q_md - q_mu) * S.geo_dyrm + (q_nd - q_nu) * S.geo_dxm[c]) * dt
                         : ((q_md - q_mu) * S.dy + (q_nd - q_nu) * S.dx) * dt;
      if (S.precip || S.use_qext) {
        float dzsdt = 0.0f;
        if (S.precip) {
          const float qinfmap = inf_cell ? qinf_cell : ((S.infiltration && v_old > 0.0) ? qi : 0.0f);  // sfincs_infiltration.f90:639-670
          dzsdt = dzsdt + (netr - qinfmap);
        }
        if (S.use_qext) dzsdt = dzsdt + qx;
        dvol = dvol + dzsdt * area * dt;
      }
      const double v = v_old + (double)dvol;
      if (v != v_old) S.zvol[c] = v;
      const float zs11 = zs_old;
      if (v >= (double)(volmax * 0.999f)) {
        zsn = (float)((double)fmaxf(S.zz_max[c], -20.0f) + (v - (double)volmax) / (double)area);
      } else if (v <= (double)1.0e-6f) {
        zsn = fmaxf(S.zz_min[c], -20.0f);
      } else {
        const float dzvol = volmax / (float)(S.nlev - 1);
        const int iuv = lev_index(v / (double)dzvol, S.nlev);
        const float facint = (float)((v - (double)((float)(iuv - 1) * dzvol)) / (double)dzvol);
        const float2 dep = S.zlev[(int64_t)(iuv - 1) * S.nalloc + c];
        zsn = dep.x + dep.y * facint;
      }
      if (zsn != zs_old) S.zs[c] = zsn;
      if (S.wiggle) {
        if (zs11 != zs00) S.zs0[c] = zs11;
        S.zsderv[c] = zsn - 2.0f * zs11 + zs00;
      }
      const uint8_t vn = v < 0.0 ? 1 : 0;
      if (vn != vn_old) S.vneg[c] = vn;
    } else {  // sfincs_continuity.f90:112-153
      float z = zs_old;
      if (S.precip) {
        const float qinfmap = inf_cell ? qinf_cell : ((S.infiltration && !(z <= zbc)) ? qi : 0.0f);
        z = z + (netr - qinfmap) * dt;
      }
      if (S.use_qext) z = z + qx * dt;
      if (S.geo)  // the cell's width, divided as the reference divides (:135-147)
        z = z + ((q_md - q_mu) / S.geo_dxm[c] + (q_nd - q_nu) * S.dyinv) * dt;
      else
        z = z + ((q_md - q_mu) * S.dxinv + (q_nd - q_nu) * S.dyinv) * dt;
      if (z != zs_old) S.zs[c] = z;
      zsn = z;
    }
    if (S.store_vmax | S.store_qmax | S.store_twet) {
      float u_md = 0.0f, u_mu = 0.0f, u_nd = 0.0f, u_nu = 0.0f;
      if (S.store_vmax) {
        u_md = S.uu[p1][c - ld];
        u_mu = S.uu[p1][c];
        u_nd = S.vv[p1][c - 1];
        u_nu = S.vv[p1][c];
      }
      store_cell_variables(S, c, q_md, q_mu, q_nd, q_nu, u_md, u_mu, u_nd, u_nu, zsn,
                           S.store_twet ? (SG ? S.zz_min[c] : S.zb[c]) : 0.0f, dt);
    }
  }
  if (S.store_zsmax) {
    if (S.store_tzsmax) store_tzsmax(S, c, zsn, zm, SG ? S.zz_min[c] : S.zb[c]);
    if (zsn > zm) S.zsmax[c] = zsn;
  }
}

// --------------------------------------------------------------------------
// Host-callable launchers.
// --------------------------------------------------------------------------
// One CTA per scenario: a thread per boundary item up to 1024 (bnd_blocks
// counts the items in 128s), one warp without boundary items.  Fewer warps
// shorten the inflow reduction: 512 instead of 1024 threads for the 400 faces
// of a 500x400 grid took its step from 15.8 to 15.4 us.
void launch_step_bnd(const ScnDev* d_scns, int nscn, int bnd_blocks, cudaStream_t s, const ScnDev* one) {
  const int threads = bnd_blocks >= 1 ? std::min(1024, bnd_blocks * 128) : 32;
  static const ScnDev none{};
  if (one)
    launch_pdl(k_step_bnd<true>, dim3(1), dim3(threads), 0, s, d_scns, *one);
  else
    launch_pdl(k_step_bnd<false>, dim3(nscn), dim3(threads), 0, s, d_scns, none);
}

// variant: CTAs per SM the register allocation is sized for (2: no spills, 3: 40 registers)
void launch_momentum(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, int variant,
                     cudaStream_t s) {
  if (ntiles <= 0) return;
  const dim3 blk(32, 8, 2);
  if (subgrid) {
    if (variant == 3)
      launch_pdl(k_momentum<true, 3>, dim3(ntiles), dim3(blk), 0, s, d_scns, d_tiles);
    else
      launch_pdl(k_momentum<true, 2>, dim3(ntiles), dim3(blk), 0, s, d_scns, d_tiles);
  } else {
    if (variant == 3)
      launch_pdl(k_momentum<false, 3>, dim3(ntiles), dim3(blk), 0, s, d_scns, d_tiles);
    else
      launch_pdl(k_momentum<false, 2>, dim3(ntiles), dim3(blk), 0, s, d_scns, d_tiles);
  }
}

void launch_sources(const ScnDev* d_scns, int nscn, cudaStream_t s) {
  launch_pdl(k_sources, dim3(nscn), dim3(32), 0, s, d_scns);
}

void launch_structures(const ScnDev* d_scns, int nscn, cudaStream_t s) {
  launch_pdl(k_structures, dim3(nscn), dim3(128), 0, s, d_scns);
}

void launch_continuity(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, cudaStream_t s) {
  if (ntiles <= 0) return;
  const dim3 blk(32, 8);
  if (subgrid)
    launch_pdl(k_continuity<true>, dim3(ntiles), dim3(blk), 0, s, d_scns, d_tiles);
  else
    launch_pdl(k_continuity<false>, dim3(ntiles), dim3(blk), 0, s, d_scns, d_tiles);
}

void launch_step(const ScnDev* d_scns, int nscn, int bnd_blocks, const Tile* d_tiles, int ntiles, int subgrid,
                 int any_src, int variant, cudaStream_t s) {
  launch_step_bnd(d_scns, nscn, bnd_blocks, s, nullptr);
  launch_momentum(d_scns, d_tiles, ntiles, subgrid, variant, s);
  if (any_src) launch_sources(d_scns, nscn, s);
  launch_continuity(d_scns, d_tiles, ntiles, subgrid, s);
}

}  // namespace sfg
