// Quadtree kernels (sm_100a): one thread per uv point (momentum), per
// combined uv point, and per cell (continuity), over compact arrays in the
// reference's order.  Work items are 256-wide chunks of one model's points
// (Tile{scenario, first, count}), so one launch advances every model of an
// ensemble.  The face arithmetic is face_flux_geo (face_math.h), shared with
// the regular-grid tile kernels; only the spacing changes per refinement
// level and at level transitions (sfincs_momentum.f90:205-313).
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "face_math.h"
#include "pdl.h"
#include "sfg_device.h"

namespace sfg {

namespace {

__device__ __forceinline__ float qt_warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace

// Momentum of one uv point per thread (sfincs_momentum.f90:157-752, quadtree
// branches).  Dry points get q = uv = 0; points that are not momentum points
// (kcuv 0, boundary faces) are left alone.
// MET: gridded wind or pressure fields (a separate instance, so that the
// plain path keeps its register allocation)
template <bool SG, bool MET>
__global__ void __launch_bounds__(256) k_qt_momentum(const ScnDev* __restrict__ scns, const Tile* __restrict__ tiles) {
  // The point's two cells, flags and table bounds are static: they are read
  // before the wait for the previous kernel, so the first round of loads after
  // it is the cell levels.  The rest of the record (the neighbour indices, in
  // the same cache lines) and the neighbours' fluxes and velocities are read
  // only for wet points: holding the whole record across the wait, or reading
  // the neighbours of every point, cost more than the round trip it saved.
  const Tile tl = tiles[blockIdx.x];
  const ScnDev& S = scns[tl.scn];
  const int i = tl.n0 + (int)threadIdx.x;
  const bool mine = (int)threadIdx.x < tl.m0;
  int2 cells = make_int2(0, 0);
  uint32_t info = 0;
  float2 zr = make_float2(0.0f, 0.0f);
  float zbmx = 0.0f;
  if (mine) {
    cells = *reinterpret_cast<const int2*>(&S.qface[i].nm);
    info = S.qface[i].info;
    if (SG)
      zr = S.sgz_u[i];
    else
      zbmx = S.zbmx[i];
  }
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  StepState& st = *S.st;
  if (!st.run) return;
  const StepVals sv = step_vals(st);
  const int p = sv.parity;
  const float* __restrict__ q0 = S.qu[p];
  const float* __restrict__ uv0 = S.uu[p];
  float* q1 = S.qu[p ^ 1];
  float* uv1 = S.uu[p ^ 1];
  float den = 0.0f;
  if (mine && (info & QF_ACT)) {
    const float zs_nm = S.zs[cells.x], zs_nmu = S.zs[cells.y];
    const float zsu = fmaxf(zs_nm, zs_nmu);
    const bool wet = SG ? zsu > zr.x + S.huthresh : zsu > zbmx;
    uint8_t* kfuv = S.kf[0];
    if (wet) {
      const FaceQ f = S.qface[i];
      const int L = (int)((f.info >> 8) & 15u);
      const int dir = (f.info & QF_DIR) ? 1 : 0;
      FaceGeo geo;
      if (!(f.info & QF_TRANS)) {
        geo.dxuvinv = dir == 0 ? S.lv_dxrinv[L] : S.lv_dyrinv[L];
        geo.dyuvinv = dir == 0 ? S.lv_dyrinv[L] : S.lv_dxrinv[L];
        geo.dxuv2inv = dir == 0 ? S.lv_dxr2inv[L] : S.lv_dyr2inv[L];
        geo.dyuv2inv = dir == 0 ? S.lv_dyr2inv[L] : S.lv_dxr2inv[L];
        geo.nuvisc = S.lv_nuvisc[L];
      } else {  // refinement transition: 1.5 cell spacing, no viscosity across (dxuv2inv = 0)
        geo.dxuvinv = dir == 0 ? S.lv_dxrinvc[L] : S.lv_dyrinvc[L];
        geo.dyuvinv = dir == 0 ? S.lv_dyrinv[L] : S.lv_dxrinv[L];
        geo.dxuv2inv = 0.0f;
        geo.dyuv2inv = dir == 0 ? S.lv_dyr2inv[L] : S.lv_dxr2inv[L];
        geo.nuvisc = S.lv_nuvisc_t[L];
      }
      geo.fcorio = S.fcorio;
      FaceV a{};
      a.qx_nm = q0[i];
      if (S.advection || S.coriolis || S.viscosity || S.friction2d || S.thetasmooth) {
        a.qx_nmd = q0[f.u_nmd];
        a.qx_nmu = q0[f.u_nmu];
        a.qy_nm = q0[f.v_nm];
        a.qy_nmu = q0[f.v_nmu];
        a.qy_ndm = q0[f.v_ndm];
        a.qy_ndmu = q0[f.v_ndmu];
        a.uu_nm = uv0[i];
        a.uu_nmd = uv0[f.u_nmd];
        a.uu_nmu = uv0[f.u_nmu];
        a.uu_ndm = uv0[f.u_ndm];
        a.uu_num = uv0[f.u_num];
        a.vu = (uv0[f.v_ndm] + uv0[f.v_ndmu] + uv0[f.v_nm] + uv0[f.v_nmu]) / 4.0f;
      }
      float hu, gnavg2, phi = 1.0f, zd0 = 0.0f, zd1 = 0.0f;
      bool dry0, dry1;
      if (SG) {
        const float zmin = zr.x, zmax = zr.y;
        if (zsu > zmax) {
          const float4 w = S.sgw_u[i];
          hu = w.x + zsu;
          gnavg2 = sg_gnavg2_full(w.z, w.y, w.w, zsu - zmax);
        } else {
          const SgLevel lv = sg_level(zsu, zmin, zmax, S.nlev);
          const UvRec r = S.rec_u[(int64_t)(lv.iuv - 1) * S.nalloc + i];
          hu = fmaf(r.dhavg, lv.facint, r.havg);
          gnavg2 = fmaf(r.dnrep, lv.facint, r.nrep);
          phi = fmaf(r.dpwet, lv.facint, r.pwet);
        }
        dry0 = S.vneg[f.nm] != 0;
        dry1 = S.vneg[f.nmu] != 0;
        if (S.wiggle) {
          zd0 = S.zsderv[f.nm];
          zd1 = S.zsderv[f.nmu];
        }
      } else {
        hu = fmaxf(zsu - zbmx, S.huthresh);
        gnavg2 = S.gn2[i];
        dry0 = zs_nm < S.zb[f.nm];
        dry1 = zs_nmu < S.zb[f.nmu];
      }
      float qn, un, tauw = dir == 0 ? sv.twu : sv.twv, dpatm = 0.0f;
      if (MET) face_meteo(S, sv, dir, f.nm, f.nmu, tauw, dpatm);
      const float ghu = face_flux_geo<SG>(S, sv, dir, (f.info & QF_ADV) != 0, (f.info & QF_TH) != 0, geo, kfuv[i],
                                          zs_nm, zs_nmu, hu, gnavg2, phi, a, dry0, dry1, zd0, zd1, tauw, dpatm, qn,
                                          un);
      den = fmaxf(sqrtf(ghu), fabsf(un)) * geo.dxuvinv;  // the face's own spacing (refinement level)
      q1[i] = qn;
      uv1[i] = un;
      kfuv[i] = KF_WET;
    } else {
      q1[i] = 0.0f;
      uv1[i] = 0.0f;
      kfuv[i] = 0;
    }
  }
  // CFL: largest denominator of the warp, one division and one atomicMin per warp
  den = qt_warp_max(den);
  if ((threadIdx.x & 31) == 0 && den > 0.0f) atomicMin(&st.min_dt_bits, __float_as_uint(1.0f / den));
}

// Combined uv points: mean of the two fine faces (sfincs_momentum.f90:757-779).
__global__ void __launch_bounds__(256) k_qt_cuv(const ScnDev* __restrict__ scns, const Tile* __restrict__ tiles) {
  const Tile tl = tiles[blockIdx.x];
  const ScnDev& S = scns[tl.scn];
  const int ic = tl.n0 + (int)threadIdx.x;
  const bool mine = (int)threadIdx.x < tl.m0;
  const int2 c = mine ? S.qcuv[ic] : make_int2(0, 0);  // static: read before the wait
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const StepState& st = *S.st;
  if (!st.run || !mine) return;
  const int p1 = st.parity ^ 1;
  float* q1 = S.qu[p1];
  float* uv1 = S.uu[p1];
  q1[S.npuv + ic] = (q1[c.x] + q1[c.y]) / 2.0f;
  uv1[S.npuv + ic] = (uv1[c.x] + uv1[c.y]) / 2.0f;
}

// Continuity of one cell per thread (sfincs_continuity.f90:46-262 and
// 265-624, quadtree spacing per refinement level).
// EXT: infiltration with state, cumulative sums, gridded rain, store variables
template <bool SG, bool EXT>
__global__ void __launch_bounds__(256) k_qt_continuity(const ScnDev* __restrict__ scns,
                                                        const Tile* __restrict__ tiles) {
  // the cell's static inputs (flags, uv points, level, volume bound) are read
  // before the wait for the previous kernel
  const Tile tl = tiles[blockIdx.x];
  const ScnDev& S = scns[tl.scn];
  const int c = tl.n0 + (int)threadIdx.x;
  const bool mine = (int)threadIdx.x < tl.m0;
  uint16_t fl = 0;
  int4 fc = make_int4(0, 0, 0, 0);
  int L = 0;
  float volmax = 0.0f;
  if (mine) {
    fl = S.flags[c];
    fc = S.qcell[c];
    L = S.qlev[c];
    if (SG) volmax = S.zz_volmax[c];
  }
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  const StepState& st = *S.st;
  if (!st.run || !mine) return;
  if (!(fl & F_ACT)) return;
  const float* q = S.qu[st.parity ^ 1];
  const float zs_old = S.zs[c];
  const float dt = st.dt;
  float zsn = zs_old;
  // infiltration with state (or cumulative rain) for every active cell, from the start-of-step state
  const bool inf_cell = EXT && S.precip && (S.inftype >= 2 || S.store_cumprcp);
  float qinf_cell = 0.0f;
  // rain of the cell: uniform from a time series, or from the gridded field
  float prc = st.ptmp, netr = st.ptmp;
  if (EXT && S.prcp_field)
    prc = cell_rain(S, c, meteo_weights(S, st.t, st.meteo_t0, st.meteo_t1), SG ? S.zvol[c] <= 0.0 : zs_old <= S.zb[c],
                    netr);
  if (inf_cell) {
    if (SG) {
      const double v0 = S.zvol[c];
      qinf_cell = cell_infiltration(S, c, prc, dt, v0 <= 0.0, (float)(v0 / (double)S.lv_area[S.qlev[c]]), st.ga_hs);
    } else {
      const float zb0 = S.zb[c];
      qinf_cell = cell_infiltration(S, c, prc, dt, zs_old <= zb0, (float)((double)zs_old - (double)zb0), st.ga_hs);
    }
  }
  if (EXT && S.qinfmap) store_qinfmap(S, c, inf_cell, qinf_cell, SG ? S.zvol[c] > 0.0 : !(zs_old <= S.zb[c]));
  if (fl & F_KCS1) {
    const float q_md = q[fc.x], q_mu = q[fc.y], q_nd = q[fc.z], q_nu = q[fc.w];
    const float qx = S.use_qext ? S.qext[c] : 0.0f;
    const float qi = S.infiltration ? S.qinf[c] : 0.0f;
    if (SG) {
      const double v_old = S.zvol[c];
      const float area = S.lv_area[L];
      const float zs00 = S.wiggle ? S.zs0[c] : 0.0f;
      float dvol = ((q_md - q_mu) * S.lv_dyrm[L] + (q_nd - q_nu) * S.lv_dxrm[L]) * dt;
      if (S.precip || S.use_qext) {
        float dzsdt = 0.0f;
        if (S.precip) {
          const float qinfmap = inf_cell ? qinf_cell : ((S.infiltration && v_old > 0.0) ? qi : 0.0f);
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
        const float2 dep = S.zlev[(int64_t)(iuv - 1) * S.npc + c];
        zsn = dep.x + dep.y * facint;
      }
      if (zsn != zs_old) S.zs[c] = zsn;
      if (S.wiggle) {
        if (zs11 != zs00) S.zs0[c] = zs11;
        S.zsderv[c] = zsn - 2.0f * zs11 + zs00;
      }
      S.vneg[c] = v < 0.0 ? 1 : 0;
    } else {
      float z = zs_old;
      if (S.precip) {
        const float zbc = S.infiltration ? S.zb[c] : 0.0f;
        const float qinfmap = inf_cell ? qinf_cell : ((S.infiltration && !(z <= zbc)) ? qi : 0.0f);
        z = z + (netr - qinfmap) * dt;
      }
      if (S.use_qext) z = z + qx * dt;
      z = z + ((q_md - q_mu) * S.lv_dxrinv[L] + (q_nd - q_nu) * S.lv_dyrinv[L]) * dt;
      if (z != zs_old) S.zs[c] = z;
      zsn = z;
    }
    if (EXT && (S.store_vmax | S.store_qmax | S.store_twet)) {
      float u_md = 0.0f, u_mu = 0.0f, u_nd = 0.0f, u_nu = 0.0f;
      if (S.store_vmax) {  // this step's velocities at the cell's uv points (combined points included)
        const float* uv = S.uu[st.parity ^ 1];
        u_md = uv[fc.x];
        u_mu = uv[fc.y];
        u_nd = uv[fc.z];
        u_nu = uv[fc.w];
      }
      store_cell_variables(S, c, q_md, q_mu, q_nd, q_nu, u_md, u_mu, u_nd, u_nu, zsn,
                           S.store_twet ? (SG ? S.zz_min[c] : S.zb[c]) : 0.0f, dt);
    }
  }
  if (S.store_zsmax) {
    const float zm = S.zsmax[c];
    if (EXT && S.store_tzsmax) store_tzsmax(S, c, zsn, zm, SG ? S.zz_min[c] : S.zb[c]);
    if (zsn > zm) S.zsmax[c] = zsn;
  }
}

void launch_qt_momentum(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, bool met, cudaStream_t s) {
  if (ntiles <= 0) return;
  auto k = subgrid ? (met ? k_qt_momentum<true, true> : k_qt_momentum<true, false>)
                   : (met ? k_qt_momentum<false, true> : k_qt_momentum<false, false>);
  launch_pdl(k, dim3(ntiles), dim3(256), 0, s, d_scns, d_tiles);
}
void launch_qt_cuv(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, cudaStream_t s) {
  if (ntiles > 0) launch_pdl(k_qt_cuv, dim3(ntiles), dim3(256), 0, s, d_scns, d_tiles);
}
void launch_qt_continuity(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, bool ext,
                          cudaStream_t s) {
  if (ntiles <= 0) return;
  auto k = subgrid ? (ext ? k_qt_continuity<true, true> : k_qt_continuity<true, false>)
                   : (ext ? k_qt_continuity<false, true> : k_qt_continuity<false, false>);
  launch_pdl(k, dim3(ntiles), dim3(256), 0, s, d_scns, d_tiles);
}

}  // namespace sfg
