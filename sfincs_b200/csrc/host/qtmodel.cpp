// Quadtree meshes: the reference's netCDF quadtree file (qtrfile) -> compact
// cells and uv points for the quadtree face/cell kernels (kernels_qt.cu).
//
// The mesh is built as the reference builds it (sfincs_domain.f90:143-1586,
// quadtree branches): active cells in quadtree order, uv points per cell (its
// right face(s), then its upper face(s)), combined uv points where a coarse
// cell borders two fine ones, the eight uv neighbours of every uv point, and
// per-level spacings.  Indices are 1-based while building (as in the
// reference) and stored 0-based; q index npuv + ncuv is the dummy point that
// stays zero.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "inputs.h"
#include "model.h"

namespace sfg {

namespace {

bool none(const std::string& s) { return s.size() >= 4 && s.compare(0, 4, "none") == 0; }

int64_t qt_key(int level, int64_t m, int64_t n) { return ((int64_t)level << 56) | (m << 28) | n; }

struct QtFile {
  long np = 0;
  int nlev = 1, nmax = 0, mmax = 0;
  float x0 = 0, y0 = 0, dx = 0, dy = 0, rot = 0;
  std::vector<int32_t> n, m, md1, md2, mu1, mu2, nd1, nd2, nu1, nu2;
  std::vector<int8_t> level, md, mu, nd, nu, mask;
  std::vector<float> z;
};

// quadtree_read_file_netcdf + quadtree_read_file: sfincs_quadtree.F90:64-160, 295-440
QtFile read_qtr(const std::string& path) {
  NcFile nc(path);
  QtFile q;
  q.np = (long)nc.dim("mesh2d_nFaces");
  auto i32 = [&](const char* v) {
    auto d = nc.doubles(v);
    return std::vector<int32_t>(d.begin(), d.end());
  };
  auto i8 = [&](const char* v) {
    auto d = nc.doubles(v);
    std::vector<int8_t> o(d.size());
    for (size_t i = 0; i < d.size(); i++) o[i] = (int8_t)d[i];
    return o;
  };
  q.n = i32("n");
  q.m = i32("m");
  q.level = i8("level");
  q.md = i8("md"), q.md1 = i32("md1"), q.md2 = i32("md2");
  q.mu = i8("mu"), q.mu1 = i32("mu1"), q.mu2 = i32("mu2");
  q.nd = i8("nd"), q.nd1 = i32("nd1"), q.nd2 = i32("nd2");
  q.nu = i8("nu"), q.nu1 = i32("nu1"), q.nu2 = i32("nu2");
  q.z = nc.floats("z");
  q.mask = i8("mask");
  q.x0 = (float)nc.att("x0");
  q.y0 = (float)nc.att("y0");
  q.dx = (float)nc.att("dx");
  q.dy = (float)nc.att("dy");
  q.rot = (float)nc.att("rotation");
  q.nmax = (int)nc.att("nmax");
  q.mmax = (int)nc.att("mmax");
  q.nlev = (int)nc.att("nr_levels");
  for (long i = 0; i < q.np; i++) {  // :118-126
    const int iref = q.level[i];
    if (iref < 1 || iref > q.nlev) throw std::runtime_error("quadtree level out of range in " + path);
    q.nmax = std::max(q.nmax, (int)((1.0f * (q.n[i] - 1) + 0.01f) / (float)(1 << (iref - 1))) + 1);
    q.mmax = std::max(q.mmax, (int)((1.0f * (q.m[i] - 1) + 0.01f) / (float)(1 << (iref - 1))) + 1);
  }
  return q;
}

}  // namespace

// Builds a HostModel of a quadtree mesh; arrays are 1-based while building.
struct QtBuilder {
  HostModel& h;
  const Keys& k;
  QtFile q;
  float rotation = 0, cosrot = 1, sinrot = 0;
  int nref = 1;
  long np = 0, npuv = 0, ncuv = 0;
  int32_t dummy = 0;
  std::vector<int32_t> sf_of_q, q_of_sf;
  std::vector<int8_t> kcs, iref_of, fmd, fmu, fnd, fnu;
  std::vector<int32_t> md1, md2, mu1, mu2, nd1, nd2, nu1, nu2;
  std::vector<int32_t> cuv_md, cuv_mu, cuv_nd, cuv_nu, cuv_uv, cuv_uv1, cuv_uv2;
  std::vector<int32_t> zuv_md, zuv_mu, zuv_nd, zuv_nu, zuv_mu1, zuv_mu2, zuv_nu1, zuv_nu2;
  std::vector<int32_t> uv_nm, uv_nmu;
  std::vector<int8_t> uv_iref, uv_dir, uv_type, kcuv;
  std::vector<int32_t> u_nmd, u_nmu, u_ndm, u_num, v_ndm, v_nm, v_ndmu, v_nmu;
  std::vector<float> dxr, dyr, zb, zbuv, sg_dep;
  QtBuilder(HostModel& hh, const Keys& kk) : h(hh), k(kk) {}
  void mesh();
  void neighbours();
  void geometry();
  void bed();
  void boundaries();
  void finish();
};

void QtBuilder::mesh() {
  ScnDev& P = h.p;
  auto path = [&](const std::string& f) { return h.dir + "/" + f; };
  if (k.qtrfile.find(".nc") == std::string::npos)
    throw std::runtime_error("only netCDF quadtree files (qtrfile *.nc) are supported");
  if (!none(k.manningfile)) throw std::runtime_error("manningfile on quadtree meshes is not supported by this core");
  q = read_qtr(path(k.qtrfile));
  if (q.nlev > kMaxQtLevels) throw std::runtime_error("more than 8 quadtree refinement levels");
  P.quadtree = 1;
  const float pi_q = 3.141592653589793f;
  rotation = q.rot * pi_q / 180.0f;
  cosrot = std::cos(rotation);
  sinrot = std::sin(rotation);
  nref = q.nlev;
  P.nref = nref;
  P.nmax = q.nmax;
  P.mmax = q.mmax;
  P.dx = q.dx;
  P.dy = q.dy;

  // ---- active cells (sfincs_domain.f90:327-482) ------------------------------------
  sf_of_q.assign((size_t)q.np + 1, 0);
  q_of_sf.assign(1, 0);
  for (long ip = 1; ip <= q.np; ip++)
    if (q.mask[ip - 1] > 0) {
      q_of_sf.push_back((int32_t)ip);
      sf_of_q[ip] = (int32_t)(q_of_sf.size() - 1);
    }
  np = (long)q_of_sf.size() - 1;
  h.np = np;
  h.qt_n = q.n;
  h.qt_m = q.m;
  h.qt_lev.assign(q.level.begin(), q.level.end());
  h.qt_nm.assign(sf_of_q.begin() + 1, sf_of_q.end());
  if (np == 0) throw std::runtime_error("quadtree mask has no active cells");
  for (auto* v : {&kcs, &iref_of, &fmd, &fmu, &fnd, &fnu}) v->assign(np + 1, 0);
  for (auto* v : {&md1, &md2, &mu1, &mu2, &nd1, &nd2, &nu1, &nu2}) v->assign(np + 1, 0);
  auto sf = [&](int32_t qi) { return qi > 0 ? sf_of_q[qi] : 0; };
  for (long nm = 1; nm <= np; nm++) {
    const long iq = q_of_sf[nm];
    kcs[nm] = q.mask[iq - 1];
    if (kcs[nm] == 4) throw std::runtime_error("msk value 4 (wave makers) is not supported");
    iref_of[nm] = q.level[iq - 1];
    fmd[nm] = q.md[iq - 1], fmu[nm] = q.mu[iq - 1], fnd[nm] = q.nd[iq - 1], fnu[nm] = q.nu[iq - 1];
    md1[nm] = sf(q.md1[iq - 1]), md2[nm] = sf(q.md2[iq - 1]);
    mu1[nm] = sf(q.mu1[iq - 1]), mu2[nm] = sf(q.mu2[iq - 1]);
    nd1[nm] = sf(q.nd1[iq - 1]), nd2[nm] = sf(q.nd2[iq - 1]);
    nu1[nm] = sf(q.nu1[iq - 1]), nu2[nm] = sf(q.nu2[iq - 1]);
    h.z_n.push_back(q.n[iq - 1]);
    h.z_m.push_back(q.m[iq - 1]);
  }
  // ---- uv points (sfincs_domain.f90:486-1003) ----------------------------------------
  long npu = 0, npv = 0;
  for (long nm = 1; nm <= np; nm++) {
    npu += (mu1[nm] > 0) + (fmu[nm] >= 1 && mu2[nm] > 0);
    npv += (nu1[nm] > 0) + (fnu[nm] >= 1 && nu2[nm] > 0);
  }
  npuv = npu + npv;
  ncuv = 0;
  for (auto* v : {&cuv_md, &cuv_mu, &cuv_nd, &cuv_nu}) v->assign(np + 1, 0);
  if (nref > 1) {  // :537-678
    for (long nm = 1; nm <= np; nm++) {
      if (fmd[nm] == 1 && (md1[nm] > 0 || md2[nm] > 0)) cuv_md[nm] = (int32_t)++ncuv;
      if (fmu[nm] == 1 && (mu1[nm] > 0 || mu2[nm] > 0)) cuv_mu[nm] = (int32_t)++ncuv;
      if (fnd[nm] == 1 && (nd1[nm] > 0 || nd2[nm] > 0)) cuv_nd[nm] = (int32_t)++ncuv;
      if (fnu[nm] == 1 && (nu1[nm] > 0 || nu2[nm] > 0)) cuv_nu[nm] = (int32_t)++ncuv;
    }
  }
  dummy = (int32_t)(npuv + ncuv + 1);  // 1-based dummy uv point
  cuv_uv.assign(ncuv + 1, 0);
  cuv_uv1.assign(ncuv + 1, dummy);
  cuv_uv2.assign(ncuv + 1, dummy);
  for (long i = 1; i <= ncuv; i++) cuv_uv[i] = (int32_t)(npuv + i);
  for (auto* v : {&zuv_md, &zuv_mu, &zuv_nd, &zuv_nu}) v->assign(np + 1, dummy);
  for (auto* v : {&zuv_mu1, &zuv_mu2, &zuv_nu1, &zuv_nu2}) v->assign(np + 1, 0);
  uv_nm.assign(npuv + 1, 0);
  uv_nmu.assign(npuv + 1, 0);
  uv_iref.assign(npuv + 1, 0);
  uv_dir.assign(npuv + 1, 0);
  uv_type.assign(npuv + 1, 0);
  long ip = 0;
  // one side (right: dir 0, upper: dir 1) of cell nm, as in :727-1003
  auto side = [&](long nm, int dir) {
    const int8_t fl = dir == 0 ? fmu[nm] : fnu[nm];
    const int32_t n1 = dir == 0 ? mu1[nm] : nu1[nm], n2 = dir == 0 ? mu2[nm] : nu2[nm];
    std::vector<int32_t>& zuv_out = dir == 0 ? zuv_mu : zuv_nu;    // this cell's side
    std::vector<int32_t>& zuv_in = dir == 0 ? zuv_md : zuv_nd;     // the neighbour's opposite side
    std::vector<int32_t>& zuv_o1 = dir == 0 ? zuv_mu1 : zuv_nu1;
    std::vector<int32_t>& zuv_o2 = dir == 0 ? zuv_mu2 : zuv_nu2;
    const std::vector<int32_t>& cuv_in = dir == 0 ? cuv_md : cuv_nd;
    const std::vector<int32_t>& cuv_out = dir == 0 ? cuv_mu : cuv_nu;
    const std::vector<int32_t>& nb1_of = dir == 0 ? md1 : nd1;  // neighbour's first opposite neighbour
    auto add = [&](int32_t other, int8_t type, int8_t lev) {
      ip++;
      uv_nm[ip] = (int32_t)nm;
      uv_nmu[ip] = other;
      uv_iref[ip] = lev;
      uv_dir[ip] = (int8_t)dir;
      uv_type[ip] = type;
    };
    if (fl == 0) {
      if (n1 > 0) {
        add(n1, 0, iref_of[nm]);
        zuv_out[nm] = (int32_t)ip;
        zuv_in[n1] = (int32_t)ip;
        zuv_o1[nm] = (int32_t)ip;
      }
    } else if (fl == -1) {  // coarser neighbour
      if (n1 > 0) {
        add(n1, -1, iref_of[nm]);
        zuv_out[nm] = (int32_t)ip;
        zuv_o1[nm] = (int32_t)ip;
        const int32_t icuv = cuv_in[n1];
        if (nb1_of[n1] == nm)
          cuv_uv1[icuv] = (int32_t)ip;
        else
          cuv_uv2[icuv] = (int32_t)ip;
        zuv_in[n1] = cuv_uv[icuv];
      }
    } else {  // two finer neighbours
      if (n1 > 0) {
        add(n1, 1, (int8_t)(iref_of[nm] + 1));
        zuv_o1[nm] = (int32_t)ip;
        zuv_in[n1] = (int32_t)ip;
        zuv_out[nm] = cuv_uv[cuv_out[nm]];
        cuv_uv1[cuv_out[nm]] = (int32_t)ip;
      }
      if (n2 > 0) {
        add(n2, 1, (int8_t)(iref_of[nm] + 1));
        zuv_o2[nm] = (int32_t)ip;
        zuv_in[n2] = (int32_t)ip;
        zuv_out[nm] = cuv_uv[cuv_out[nm]];
        cuv_uv2[cuv_out[nm]] = (int32_t)ip;
      }
    }
  };
  for (long nm = 1; nm <= np; nm++) {
    side(nm, 0);
    side(nm, 1);
  }
  if (ip != npuv) throw std::runtime_error("quadtree uv point count mismatch");
  h.npuv = npuv;
}

// Eight uv neighbours of every uv point (sfincs_domain.f90:1007-1261), with
// the reference's fill-ins: missing u neighbours point at the uv point itself,
// missing v neighbours at the dummy point.
void QtBuilder::neighbours() {
  for (auto* v : {&u_nmd, &u_nmu, &u_ndm, &u_num, &v_ndm, &v_nm, &v_ndmu, &v_nmu}) v->assign(npuv + 1, 0);
  for (long ip = 1; ip <= npuv; ip++) {
    const long nm = uv_nm[ip];
    if (uv_dir[ip] == 0) {
      const long nmu = uv_nmu[ip];
      u_nmd[ip] = zuv_md[nm];
      u_nmu[ip] = zuv_mu[nmu];
      if (fnd[nm] > -1) {
        const long ndm = nd1[nm];
        if (ndm > 0) u_ndm[ip] = zuv_mu[ndm];
      } else {
        const long ndm = nd2[nm];
        if (ndm > 0) {
          if (fmu[ndm] == 0) {
            u_ndm[ip] = zuv_mu[ndm];
          } else {
            const long ndmu = mu1[ndm];
            if (ndmu > 0) u_ndm[ip] = zuv_md[ndmu];
          }
        }
      }
      if (fnu[nm] > -1) {
        const long num = nu1[nm];
        if (num > 0) u_num[ip] = zuv_mu[num];
      } else {
        const long num = nu2[nm];
        if (num > 0) {
          if (fmu[num] == 0) {
            u_num[ip] = zuv_mu[num];
          } else {
            const long numu = mu1[num];
            if (numu > 0) u_num[ip] = zuv_md[numu];
          }
        }
      }
      v_nm[ip] = zuv_nu[nm];
      v_ndm[ip] = zuv_nd[nm];
      v_nmu[ip] = zuv_nu[nmu];
      v_ndmu[ip] = zuv_nd[nmu];
    } else {
      const long num = uv_nmu[ip];
      u_nmd[ip] = zuv_nd[nm];
      u_nmu[ip] = zuv_nu[num];
      if (fmd[nm] > -1) {
        const long nmd = md1[nm];
        if (nmd > 0) u_ndm[ip] = zuv_nu[nmd];
      } else {
        const long nmd = md2[nm];
        if (nmd > 0) {
          if (fnu[nmd] == 0) {
            u_ndm[ip] = zuv_nu[nmd];
          } else {
            const long nmdu = nu1[nmd];
            if (nmdu > 0) u_ndm[ip] = zuv_nd[nmdu];
          }
        }
      }
      if (fmu[nm] > -1) {
        const long nmu = mu1[nm];
        if (nmu > 0) u_num[ip] = zuv_nu[nmu];
      } else {
        const long nmu = mu2[nm];
        if (nmu > 0) {
          if (fnu[nmu] == 0) {
            u_num[ip] = zuv_nu[nmu];
          } else {
            const long numu = nu1[nmu];
            if (numu > 0) u_num[ip] = zuv_nd[numu];
          }
        }
      }
      v_nm[ip] = zuv_mu[nm];
      v_ndm[ip] = zuv_md[nm];
      v_nmu[ip] = zuv_mu[num];
      v_ndmu[ip] = zuv_md[num];
    }
    if (u_nmd[ip] == 0) u_nmd[ip] = (int32_t)ip;
    if (u_nmu[ip] == 0) u_nmu[ip] = (int32_t)ip;
    if (u_ndm[ip] == 0) u_ndm[ip] = (int32_t)ip;
    if (u_num[ip] == 0) u_num[ip] = (int32_t)ip;
    if (v_ndm[ip] == 0) v_ndm[ip] = dummy;
    if (v_ndmu[ip] == 0) v_ndmu[ip] = dummy;
    if (v_nm[ip] == 0) v_nm[ip] = dummy;
    if (v_nmu[ip] == 0) v_nmu[ip] = dummy;
  }
}

// Per-level spacing, cell centres, time-step limits and viscosity
// (sfincs_domain.f90:1369-1541, projected coordinates).
void QtBuilder::geometry() {
  ScnDev& P = h.p;
  dxr.assign(nref + 1, 0.0f);
  dyr.assign(nref + 1, 0.0f);
  float dxymin = 1.0e6f;
  for (int i = 1; i <= nref; i++) {
    dxr[i] = q.dx / (float)(1 << (i - 1));
    dyr[i] = q.dy / (float)(1 << (i - 1));
    const int L = i - 1;
    P.lv_dxrm[L] = dxr[i];
    P.lv_dxrinv[L] = 1.0f / P.lv_dxrm[L];
    P.lv_dxr2inv[L] = P.lv_dxrinv[L] * P.lv_dxrinv[L];
    P.lv_dyrm[L] = dyr[i];
    P.lv_dyrinv[L] = 1.0f / P.lv_dyrm[L];
    P.lv_dyr2inv[L] = P.lv_dyrinv[L] * P.lv_dyrinv[L];
    P.lv_area[L] = P.lv_dxrm[L] * P.lv_dyrm[L];
    if (i > 1) {
      P.lv_dxrinvc[L] = 1.0f / (3.0f * P.lv_dxrm[L] / 2.0f);
      P.lv_dyrinvc[L] = 1.0f / (3.0f * P.lv_dyrm[L] / 2.0f);
    }
    dxymin = std::min(dxymin, dxr[i]);
    dxymin = std::min(dxymin, dyr[i]);
    P.lv_nuvisc[L] = k.viscosity ? std::max(k.nuviscdim * std::min(dxr[i], dyr[i]), 0.0f) : 0.0f;
    P.lv_nuvisc_t[L] = P.nuviscfac * P.lv_nuvisc[L];  // transition faces (sfincs_momentum.f90:519-527)
  }
  P.dtmax = std::min(k.dtmax, P.alfa * dxymin / (std::sqrt(9.81f * k.hmin_cfl)));
  P.dtmin = P.alfa * dxymin / (1.25f * std::fabs(k.uvmax));
  // the regular-grid fields hold the level-1 values (k_step, boundary kernels)
  P.dxinv = P.lv_dxrinv[0];
  P.dyinv = P.lv_dyrinv[0];
  P.dx2inv = P.lv_dxr2inv[0];
  P.dy2inv = P.lv_dyr2inv[0];
  P.area = P.lv_area[0];
  P.nuvisc = P.lv_nuvisc[0];
  h.qt_dxr.assign(dxr.begin() + 1, dxr.end());
  h.qt_dyr.assign(dyr.begin() + 1, dyr.end());
  h.z_xz.resize(np);
  h.z_yz.resize(np);
  h.cell_area.resize(np);
  for (long nm = 1; nm <= np; nm++) {
    const float n = (float)h.z_n[nm - 1], m = (float)h.z_m[nm - 1];
    const int i = iref_of[nm];
    h.z_xz[nm - 1] = q.x0 + cosrot * (1.0f * (m - 0.5f)) * dxr[i] - sinrot * (1.0f * (n - 0.5f)) * dyr[i];
    h.z_yz[nm - 1] = q.y0 + sinrot * (1.0f * (m - 0.5f)) * dxr[i] + cosrot * (1.0f * (n - 0.5f)) * dyr[i];
    h.cell_area[nm - 1] = P.lv_area[i - 1];
  }
  h.x0 = q.x0;
  h.y0 = q.y0;
  h.cosrot = cosrot;
  h.sinrot = sinrot;
}

// Bed level, uv bed levels and roughness (sfincs_domain.f90:1588-1744,
// 1960-2061) or the quadtree subgrid tables (sfincs_subgrid.F90:57-455).
void QtBuilder::bed() {
  ScnDev& P = h.p;
  auto path = [&](const std::string& f) { return h.dir + "/" + f; };
  h.zb_cmp.assign(np, 0.0f);
  h.zmin_cmp.assign(np, 0.0f);
  if (!P.subgrid) {
    zb.assign(np + 1, 0.0f);
    if (none(k.depfile)) {
      for (long nm = 1; nm <= np; nm++) zb[nm] = q.z[q_of_sf[nm] - 1];
    } else {
      auto d = read_binary<float>(path(k.depfile), (size_t)np);
      for (long nm = 1; nm <= np; nm++) zb[nm] = d[nm - 1];
    }
    zbuv.assign(npuv + 1, 0.0f);
    h.zbmx_q.assign(npuv, 0.0f);
    for (long ip = 1; ip <= npuv; ip++) {
      const long nm = uv_nm[ip], nmu = uv_nmu[ip];
      if (uv_type[ip] == 0)
        zbuv[ip] = 0.5f * (zb[nm] + zb[nmu]);
      else if (uv_type[ip] == -1)
        zbuv[ip] = 0.3333f * zb[nm] + 0.6667f * zb[nmu];
      else
        zbuv[ip] = 0.6667f * zb[nm] + 0.3333f * zb[nmu];
      h.zbmx_q[ip - 1] = std::max(zb[nm], zb[nmu]) + P.huthresh;
    }
    h.zb.assign(np, 0.0f);
    for (long nm = 1; nm <= np; nm++) h.zb[nm - 1] = h.zb_cmp[nm - 1] = zb[nm];
    return;
  }
  NcFile nc(path(k.sbgfile));
  const int L = (int)nc.dim("levels");
  if (L < 2) throw std::runtime_error("subgrid tables need at least two levels");
  P.nlev = L;
  auto zmin = nc.floats("z_zmin"), zmax = nc.floats("z_zmax"), volmax = nc.floats("z_volmax"),
       zlev = nc.floats("z_level"), uzmin = nc.floats("uv_zmin"), uzmax = nc.floats("uv_zmax"),
       uffit = nc.floats("uv_ffit"), unavg = nc.floats("uv_navg"), uhavg = nc.floats("uv_havg"),
       unrep = nc.floats("uv_nrep"), upwet = nc.floats("uv_pwet");
  // file index of every active cell and uv point: the file covers every
  // quadtree point and, per point, its right then upper faces (:166-245)
  std::vector<long> zi(np), ui(npuv);
  long npuvq = 0, npuvs = 0;
  for (long ip = 1; ip <= q.np; ip++) {
    const long nm = sf_of_q[ip];
    if (nm > 0) zi[nm - 1] = ip - 1;
    auto face = [&](int32_t nb, const std::vector<int32_t>& zuv) {
      if (nb > 0) {
        npuvq++;
        if (nm > 0 && zuv[nm] > 0) {
          if (npuvs >= npuv) throw std::runtime_error("subgrid file faces do not match the quadtree mesh");
          ui[npuvs++] = npuvq - 1;
        }
      }
    };
    if (q.mu[ip - 1] < 1) {
      face(q.mu1[ip - 1], zuv_mu1);
    } else {
      face(q.mu1[ip - 1], zuv_mu1);
      face(q.mu2[ip - 1], zuv_mu2);
    }
    if (q.nu[ip - 1] < 1) {
      face(q.nu1[ip - 1], zuv_nu1);
    } else {
      face(q.nu1[ip - 1], zuv_nu1);
      face(q.nu2[ip - 1], zuv_nu2);
    }
  }
  if ((long)zmin.size() != q.np || (long)uzmin.size() != npuvq || npuvs != npuv)
    throw std::runtime_error("subgrid file dimensions do not match the quadtree mesh");
  std::vector<float> czmin(np), czmax(np), fzmin(npuv), fzmax(npuv);
  for (long i = 0; i < np; i++) {
    czmin[i] = zmin[zi[i]];
    czmax[i] = zmax[zi[i]];
  }
  for (long f = 0; f < npuv; f++) {
    fzmin[f] = uzmin[ui[f]];
    fzmax[f] = std::max(uzmax[ui[f]], fzmin[f] + 0.01f);
  }
  for (long f = 0; f < npuv; f++) {  // :364-388
    const float zn = czmin[uv_nm[f + 1] - 1], znu = czmin[uv_nmu[f + 1] - 1];
    if (zn > fzmin[f]) {
      fzmin[f] = std::max(fzmin[f], zn);
      fzmax[f] = std::max(fzmax[f], fzmin[f] + 0.01f);
    }
    if (znu > fzmin[f]) {
      fzmin[f] = std::max(fzmin[f], znu);
      fzmax[f] = std::max(fzmax[f], fzmin[f] + 0.01f);
    }
  }
  for (long i = 0; i < np; i++)
    if (czmax[i] - czmin[i] <= 0.0f) czmax[i] = czmax[i] + 0.01f;
  for (long f = 0; f < npuv; f++)
    if (fzmax[f] - fzmin[f] < 1.0e-7f) fzmax[f] = fzmax[f] + 0.01f;
  h.zz_min = czmin;
  h.zz_max = czmax;
  h.zz_volmax.resize(np);
  h.zlev.assign((size_t)(L - 1) * np, make_float2(0.0f, 0.0f));
  sg_dep.assign((size_t)np * L, 0.0f);
  for (long i = 0; i < np; i++) {
    h.zz_volmax[i] = volmax[zi[i]];
    h.zmin_cmp[i] = czmin[i];
    for (int kk = 0; kk < L; kk++) sg_dep[(size_t)i * L + kk] = zlev[(size_t)zi[i] * L + kk];
    for (int kk = 0; kk < L - 1; kk++) {
      const float a = sg_dep[(size_t)i * L + kk], b = sg_dep[(size_t)i * L + kk + 1];
      h.zlev[(size_t)kk * np + i] = make_float2(a, b - a);
    }
  }
  h.sgz_u.resize(npuv);
  h.sgw_u.resize(npuv);
  h.rec_u.assign((size_t)(L - 1) * npuv, UvRec{});
  std::vector<float> hv(L), nv(L), pv(L);
  for (long f = 0; f < npuv; f++) {
    const long r = ui[f];
    for (int kk = 0; kk < L; kk++) {
      hv[kk] = uhavg[(size_t)r * L + kk];
      const float nr = std::max(unrep[(size_t)r * L + kk], 0.0001f);
      nv[kk] = P.g * (nr * nr);
      pv[kk] = upwet[(size_t)r * L + kk];
    }
    const float na = std::max(unavg[r], 0.0001f);
    h.sgz_u[f] = make_float2(fzmin[f], fzmax[f]);
    h.sgw_u[f] = make_float4(hv[L - 1] - fzmax[f], nv[L - 1], P.g * (na * na), uffit[r]);
    for (int kk = 0; kk < L - 1; kk++) {
      UvRec rr{};
      rr.havg = hv[kk];
      rr.dhavg = hv[kk + 1] - hv[kk];
      rr.nrep = nv[kk];
      rr.dnrep = nv[kk + 1] - nv[kk];
      rr.pwet = pv[kk];
      rr.dpwet = pv[kk + 1] - pv[kk];
      h.rec_u[(size_t)kk * npuv + f] = rr;
    }
  }
}

// kcuv classification, water-level boundary faces, boundary forcing files and
// boundary point weights (sfincs_domain.f90:1765-1958, sfincs_boundaries.f90:8-213, 455-679).
void QtBuilder::boundaries() {
  ScnDev& P = h.p;
  auto path = [&](const std::string& f) { return h.dir + "/" + f; };
  // point lookup keys (find_quadtree_cell: sfincs_quadtree.F90:764-820)
  {
    std::vector<std::pair<int64_t, int32_t>> kv((size_t)np);
    for (long nm = 1; nm <= np; nm++)
      kv[nm - 1] = {qt_key(iref_of[nm], h.z_m[nm - 1], h.z_n[nm - 1]), (int32_t)(nm - 1)};
    std::sort(kv.begin(), kv.end());
    h.qt_key.resize(np);
    h.qt_key_cell.resize(np);
    for (long i = 0; i < np; i++) h.qt_key[i] = kv[i].first, h.qt_key_cell[i] = kv[i].second;
  }
  // the active cell of level iref at (n, m), 0 if none (find_sfincs_cell)
  auto cell_at = [&](long n, long m, int iref) -> long {
    const int64_t key = qt_key(iref, m, n);
    auto it = std::lower_bound(h.qt_key.begin(), h.qt_key.end(), key);
    return (it != h.qt_key.end() && *it == key) ? (long)h.qt_key_cell[it - h.qt_key.begin()] + 1 : 0;
  };
  kcuv.assign(npuv + ncuv + 2, 0);
  auto kcuv_of = [](int a, int b) -> int8_t {
    if (a > 1 && b > 1) return 0;
    if (a * b == 0) return 0;
    if ((a == 1 && b == 2) || (a == 2 && b == 1)) return 2;
    if ((a == 1 && b == 3) || (a == 3 && b == 1)) return 2;
    if ((a == 1 && b == 5) || (a == 5 && b == 1)) return 2;
    if ((a == 1 && b == 6) || (a == 6 && b == 1)) return 6;
    return 1;
  };
  for (long ip = 1; ip <= npuv; ip++) kcuv[ip] = kcuv_of(kcs[uv_nm[ip]], kcs[uv_nmu[ip]]);
  // boundary cells (water level, outflow, downstream river, Neumann; sfincs_domain.f90:1786-1830) and their forcing
  std::vector<int32_t> gb_cell, gb_index(np + 1, -1);
  bool water_level_bnd = false;
  for (long nm = 1; nm <= np; nm++)
    if (kcs[nm] == 2 || kcs[nm] == 3 || kcs[nm] == 5 || kcs[nm] == 6) {
      gb_index[nm] = (int32_t)gb_cell.size();
      gb_cell.push_back((int32_t)nm);
      h.gb_cmp.push_back((int32_t)(nm - 1));
      if (kcs[nm] == 2) water_level_bnd = true;
    }
  const size_t ngb = gb_cell.size();
  std::vector<float> xb, yb;
  int nbnd = 0;
  read_boundary_series(h, k, water_level_bnd, xb, yb, nbnd);
  // downstream river points (sfincs_boundaries.f90:217-270): the cell of each
  // point's internal point and the level drop slope * distance to it
  std::vector<float> xr, yr, dzr;
  std::vector<int32_t> zsir;
  bool river = false;
  for (long nm : gb_cell) river = river || kcs[nm] == 5;
  if (river) {
    if (none(k.bdrfile)) throw std::runtime_error("downstream river points (msk 5) need a bdrfile");
    for (const auto& r : read_table(path(k.bdrfile))) {
      if (r.size() < 6) throw std::runtime_error("bdrfile: expected x y x_internal y_internal slope distance");
      const float x = (float)r[0], y = (float)r[1], xin = (float)r[2], yin = (float)r[3];
      const float slope = (float)r[4], dist = (float)r[5];
      const int ci = quadtree_cell_index(h, xin, yin);
      if (ci <= 0) throw std::runtime_error("bdrfile: internal point outside the active mesh");
      xr.push_back(x);
      yr.push_back(y);
      zsir.push_back(ci - 1);
      dzr.push_back(dist < 0.0f ? -slope * std::sqrt((xin - x) * (xin - x) + (yin - y) * (yin - y)) : -slope * dist);
    }
    if (xr.empty()) throw std::runtime_error("bdrfile holds no points");
  }
  std::vector<int> gb_bdr(ngb, -1);
  for (size_t ib = 0; ib < ngb; ib++) {
    const long nm = gb_cell[ib];
    if (kcs[nm] == 5) {  // nearest point of the bdr file (:596-613)
      const float x = h.z_xz[nm - 1], y = h.z_yz[nm - 1];
      float dst1 = 1.0e10f;
      for (size_t j = 0; j < xr.size(); j++) {
        const float ddx = xr[j] - x, ddy = yr[j] - y;
        const float dst = std::sqrt(ddx * ddx + ddy * ddy);
        if (dst < dst1) {
          dst1 = dst;
          gb_bdr[ib] = (int)j;
        }
      }
    } else if (kcs[nm] == 6) {  // Neumann: the last regular neighbour of the same level found (:615-672)
      const long n = h.z_n[nm - 1], m = h.z_m[nm - 1];
      const int iref = iref_of[nm];
      const long cand[4][2] = {{n, m + 1}, {n + 1, m}, {n, m - 1}, {n - 1, m}};
      long nmi = 0;
      for (auto& c : cand) {
        const long ci = cell_at(c[0], c[1], iref);
        if (ci > 0 && kcs[ci] == 1) nmi = ci;
      }
      if (nmi == 0)
        kcs[nm] = 0;  // isolated Neumann cell reset to inactive
      else
        h.neu.push_back(make_int2((int)(nm - 1), (int)(nmi - 1)));
    }
  }
  std::vector<int> gb_i1(ngb, 0), gb_i2(ngb, 0);
  std::vector<float> gb_fac(ngb, 0.0f);
  if (nbnd > 0)
    for (size_t ib = 0; ib < ngb; ib++) {
      const long nm = gb_cell[ib];
      if (kcs[nm] != 2) continue;
      if (nbnd > 1) {
        const float x = h.z_xz[nm - 1], y = h.z_yz[nm - 1];
        float dst1 = 1.0e10f, dst2 = 1.0e10f;
        int ib1 = 0, ib2 = 0;
        for (int j = 0; j < nbnd; j++) {
          const float ddx = xb[j] - x, ddy = yb[j] - y;
          const float dst = std::sqrt(ddx * ddx + ddy * ddy);
          if (dst < dst1) {
            dst2 = dst1;
            ib2 = ib1;
            dst1 = dst;
            ib1 = j + 1;
          } else if (dst < dst2) {
            dst2 = dst;
            ib2 = j + 1;
          }
        }
        if (ib2 == 0) ib2 = ib1;
        gb_i1[ib] = ib1 - 1;
        gb_i2[ib] = ib2 - 1;
        gb_fac[ib] = dst2 / std::max(dst1 + dst2, 1.0e-9f);
      } else {
        gb_fac[ib] = 1.0f;
      }
    }
  // the reference's boundary-face list holds the faces with kcuv 2 or 6; those
  // of Neumann cells are left to the momentum kernel, but a Neumann cell reset
  // to inactive keeps its faces in the list with its level zsb at its initial
  // 0 (sfincs_boundaries.f90:661-672, 800-921, 947-960)
  for (long ip = 1; ip <= npuv; ip++) {
    if (kcuv[ip] != 2 && kcuv[ip] != 6) continue;
    const long a = uv_nm[ip], b = uv_nmu[ip];
    const bool a_int = kcs[a] == 1;
    const long nmb = a_int ? b : a, nmi = a_int ? a : b;
    if (kcuv[ip] == 6 && kcs[nmb] != 0) continue;
    BndFace f{};
    f.face = (int)(ip - 1);
    f.nmb = (int)(nmb - 1);
    f.nmi = (int)(nmi - 1);
    const int ib = gb_index[nmb];
    f.info = (uv_dir[ip] == 1 ? 1 : 0) | (a_int ? 0 : 2) | (kcs[nmb] == 3 ? 4 : 0) | (nbnd > 1 ? 8 : 0);
    f.i1 = gb_i1[ib];
    f.i2 = gb_i2[ib];
    f.fac = gb_fac[ib];
    f.zbuv = P.subgrid ? 0.0f : zbuv[ip];
    f.floor = P.subgrid ? h.zz_min[nmb - 1] : zb[nmb];
    f.zfix = kcs[nmb] == 3 ? f.floor : 0.0f;
    f.len = uv_dir[ip] == 1 ? dxr[uv_iref[ip]] : dyr[uv_iref[ip]];
    if (kcs[nmb] == 2 && nbnd == 0) f.info |= 4, f.zfix = 0.0f;  // no boundary data: zsb stays 0
    if (kcs[nmb] == 0) f.info |= 4, f.zfix = 0.0f;                 // reset Neumann cell: zsb stays 0
    if (kcs[nmb] == 5) {  // downstream river cell: level from its internal point
      const int j = gb_bdr[ib];
      if (j < 0) throw std::runtime_error("downstream river cell without a bdr point");
      f.info = (f.info & ~8) | 32;
      f.zsi = zsir[(size_t)j];
      f.zfix = dzr[(size_t)j];
      f.i1 = f.i2 = 0;
    }
    h.bfaces.push_back(f);
  }
  P.ngbnd = (int)ngb;
  P.nkcuv2 = (int)h.bfaces.size();
  P.nneu = (int)h.neu.size();
}

// Device records of the uv points and cells, advection mask, roughness,
// infiltration, initial state and meteo series.
void QtBuilder::finish() {
  ScnDev& P = h.p;
  P.npc = (int)np;
  P.npuv = (int)npuv;
  P.ncuv = (int)ncuv;
  P.nalloc = (int64_t)npuv;  // level stride of the face tables (boundary kernel)
  P.ld = 0;
  // kcuv of the combined points (set_advection_mask: sfincs_domain.f90:2114-2130)
  for (long ic = 1; ic <= ncuv; ic++) {
    const int a = kcuv[cuv_uv1[ic]], b = kcuv[cuv_uv2[ic]];
    int8_t& kk = kcuv[cuv_uv[ic]];
    if (a == 0 || b == 0)
      kk = 0;
    else if (a == 2 || b == 2)
      kk = 2;
    else if (a == 4 || b == 4)
      kk = 4;
    else
      kk = 1;
  }
  const bool do_mask = P.advection && k.advection_mask && (nref > 1 || q.nmax > 1);  // :2132-2178
  // Thin dams (sfincs_structures.f90:385-495, sfincs_quadtree.F90:853-1010):
  // per dam segment and refinement level, the cells in the segment's cell
  // index box widened by one; a right or upper uv point whose segment between
  // the two cell centres crosses the dam gets kcuv 0.  Applied after the
  // boundary lists, the combined points and the advection mask, as the
  // reference applies them after initialize_domain.
  std::vector<int8_t> kcuv_run = kcuv;
  auto path = [&](const std::string& f) { return h.dir + "/" + f; };
  // uv points crossed by one polyline -> the last segment crossing each
  auto crossed = [&](const std::vector<PolyRow>& pl) {
    std::map<long, int> ind;
    for (size_t ipol = 0; ipol + 1 < pl.size(); ipol++) {
      const float xpa = pl[ipol].x, ypa = pl[ipol].y, xpb = pl[ipol + 1].x, ypb = pl[ipol + 1].y;
      const float xta = cosrot * (xpa - q.x0) + sinrot * (ypa - q.y0), yta = -sinrot * (xpa - q.x0) + cosrot * (ypa - q.y0);
      const float xtb = cosrot * (xpb - q.x0) + sinrot * (ypb - q.y0), ytb = -sinrot * (xpb - q.x0) + cosrot * (ypb - q.y0);
      for (int iref = nref; iref >= 1; iref--) {
        const int64_t na = (int64_t)(yta / dyr[iref]) + 1, ma = (int64_t)(xta / dxr[iref]) + 1;
        const int64_t nb = (int64_t)(ytb / dyr[iref]) + 1, mb = (int64_t)(xtb / dxr[iref]) + 1;
        for (int64_t m = std::max(std::min(ma, mb) - 1, (int64_t)1); m <= std::max(ma, mb) + 1; m++) {
          for (int64_t n = std::max(std::min(na, nb) - 1, (int64_t)1); n <= std::max(na, nb) + 1; n++) {
            const int64_t key = qt_key(iref, m, n);
            auto it = std::lower_bound(h.qt_key.begin(), h.qt_key.end(), key);
            if (it == h.qt_key.end() || *it != key) continue;  // no active cell of this level here
            const long nm = h.qt_key_cell[it - h.qt_key.begin()] + 1;
            for (int32_t ip : {zuv_mu1[nm], zuv_mu2[nm], zuv_nu1[nm], zuv_nu2[nm]}) {
              if (ip <= 0) continue;
              const long nmu = uv_nmu[ip];
              if (segments_cross(xpa, ypa, xpb, ypb, h.z_xz[nm - 1], h.z_yz[nm - 1], h.z_xz[nmu - 1], h.z_yz[nmu - 1]))
                ind[ip] = (int)ipol;
            }
          }
        }
      }
    }
    return ind;
  };
  // cross-sections (sfincs_crosssections.f90:8-127): the crossed uv points in
  // uv-point order, the sign from the last segment crossing each, the width
  // of the point's refinement level
  if (!none(h.out.crsfile)) {
    std::vector<std::string> names;
    const auto pls = read_polylines(path(h.out.crsfile), 0, &names);
    for (size_t kp = 0; kp < pls.size(); kp++) {
      CrossSection cs;
      cs.name = names[kp];
      for (const auto& e : crossed(pls[kp])) {
        const long ip = e.first, nm = uv_nm[ip], nmu = uv_nmu[ip];
        const int dir = uv_dir[ip];
        const auto& a = pls[kp][(size_t)e.second];
        const auto& b = pls[kp][(size_t)e.second + 1];
        cs.faces.push_back(CrsFace{ip - 1, dir,
                                   crossing_sign(h.z_xz[nm - 1], h.z_yz[nm - 1], h.z_xz[nmu - 1], h.z_yz[nmu - 1], a.x,
                                                 a.y, b.x, b.y, h.p.pi),
                                   dir == 0 ? dyr[uv_iref[ip]] : dxr[uv_iref[ip]]});
      }
      h.out.crs.push_back(std::move(cs));
    }
  }
  if (!none(k.thdfile))
    for (const auto& pl : read_polylines(path(k.thdfile), 0))
      for (const auto& e : crossed(pl)) kcuv_run[e.first] = 0;
  // Weirs (sfincs_structures.f90:38-381): crossed length, crest and Cd per uv
  // point, kept where the crest is above the face bed (kcuv 3, after the dams)
  if (!none(k.weirfile)) {
    struct Acc {
      float len = 0.0f, height = -9999.0f, cd = 0.0f;
    };
    std::map<long, Acc> acc;
    const float pi = P.pi;
    for (const auto& pl : read_polylines(path(k.weirfile), 2)) {
      for (const auto& e : crossed(pl)) {
        const long ip = e.first, nm = uv_nm[ip], nmu = uv_nmu[ip];
        const int iref = uv_iref[ip], idir = uv_dir[ip];
        const float dxs = idir == 0 ? dyr[iref] : dxr[iref];
        float xuv, yuv, xuv1, yuv1, xuv2, yuv2;
        if (iref_of[nm] >= iref_of[nmu]) {  // normal point or fine to coarse
          xuv = h.z_xz[nm - 1] + 0.5f * dxs * std::cos(idir == 0 ? rotation : rotation + 0.5f * pi);
          yuv = h.z_yz[nm - 1] + 0.5f * dxs * std::sin(idir == 0 ? rotation : rotation + 0.5f * pi);
        } else {
          xuv = h.z_xz[nmu - 1] + 0.5f * dxs * std::cos(idir == 0 ? rotation - pi : rotation - 0.5f * pi);
          yuv = h.z_yz[nmu - 1] + 0.5f * dxs * std::sin(idir == 0 ? rotation - pi : rotation - 0.5f * pi);
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
        const PolyRow &r0 = pl[(size_t)e.second], &r1 = pl[(size_t)e.second + 1];
        Acc& a = acc[ip];
        a.len = a.len + projected_length(xuv1, yuv1, xuv2, yuv2, r0.x, r0.y, r1.x, r1.y);
        const float dst1 = std::sqrt((xuv - r0.x) * (xuv - r0.x) + (yuv - r0.y) * (yuv - r0.y));
        const float dst2 = std::sqrt((xuv - r1.x) * (xuv - r1.x) + (yuv - r1.y) * (yuv - r1.y));
        const float wfac = dst1 / (dst1 + dst2);
        a.height = std::max(a.height, r0.p[0] * (1.0f - wfac) + r1.p[0] * wfac);
        a.cd = r0.p[1] * (1.0f - wfac) + r1.p[1] * wfac;
      }
    }
    std::vector<uint8_t> weir(npuv + 2, 0);
    for (const auto& e : acc) {
      const long ip = e.first;
      const float bed = P.subgrid ? h.sgz_u[ip - 1].x : h.zbmx_q[ip - 1];
      if (!(e.second.height > bed)) continue;
      StrucFace w{};
      w.face = (int)(ip - 1);
      w.nm = (int)(uv_nm[ip] - 1);
      w.nmu = (int)(uv_nmu[ip] - 1);
      w.dir = uv_dir[ip];
      w.height = e.second.height;
      w.cd = e.second.cd;
      w.len = e.second.len / (uv_dir[ip] == 0 ? dyr[uv_iref[ip]] : dxr[uv_iref[ip]]);
      h.struc.push_back(w);
      kcuv_run[ip] = 3;
      weir[ip] = 1;
    }
    for (auto& b : h.bfaces)
      if (weir[b.face + 1]) b.info |= 16;  // no boundary flux under a weir (sfincs_boundaries.f90:1009)
  }
  P.nstruc = (int)h.struc.size();
  // roughness of regular beds (sfincs_domain.f90:1960-2061)
  if (!P.subgrid) {
    h.gn2_q.assign(npuv, 9.81f * 0.02f * 0.02f);
    const float gn2land = k.manning_land < 0.0f ? 9.81f * (k.manning * k.manning)
                                               : 9.81f * (k.manning_land * k.manning_land);
    const float gn2sea = k.manning_sea < 0.0f ? 9.81f * (k.manning * k.manning)
                                             : 9.81f * (k.manning_sea * k.manning_sea);
    for (long ip = 1; ip <= npuv; ip++)
      if (kcuv[ip] > 0) h.gn2_q[ip - 1] = zbuv[ip] > k.rghlevland ? gn2land : gn2sea;
  }
  h.qface.resize(npuv);
  for (long ip = 1; ip <= npuv; ip++) {
    FaceQ f{};
    f.nm = uv_nm[ip] - 1;
    f.nmu = uv_nmu[ip] - 1;
    f.u_nmd = u_nmd[ip] - 1, f.u_nmu = u_nmu[ip] - 1, f.u_ndm = u_ndm[ip] - 1, f.u_num = u_num[ip] - 1;
    f.v_ndm = v_ndm[ip] - 1, f.v_nm = v_nm[ip] - 1, f.v_ndmu = v_ndmu[ip] - 1, f.v_nmu = v_nmu[ip] - 1;
    uint32_t info = (uv_dir[ip] == 1 ? QF_DIR : 0u);
    if (kcuv_run[ip] == 1 || kcuv_run[ip] == 6) info |= QF_ACT;
    bool adv = P.advection;
    if (do_mask && (kcuv[u_nmu[ip]] != 1 || kcuv[u_nmd[ip]] != 1 || kcuv[v_nm[ip]] != 1 || kcuv[v_nmu[ip]] != 1 ||
                    kcuv[v_ndm[ip]] != 1 || kcuv[v_ndmu[ip]] != 1 || kcuv[u_ndm[ip]] != 1 || kcuv[u_num[ip]] != 1))
      adv = false;
    if (adv) info |= QF_ADV;
    if (kcuv_run[u_nmd[ip]] == 1 && kcuv_run[u_nmu[ip]] == 1) info |= QF_TH;
    if (uv_type[ip] != 0) info |= QF_TRANS;
    info |= (uint32_t)(uv_iref[ip] - 1) << 8;
    f.info = info;
    h.qface[ip - 1] = f;
  }
  h.qcell.resize(np);
  h.qlev.resize(np);
  h.qmap_u.resize(np);
  h.qmap_v.resize(np);
  h.flags.assign(np, 0);
  h.kcs_cmp.resize(np);
  h.cmp_off.resize(np);
  h.dense2cmp.resize(np);
  for (long nm = 1; nm <= np; nm++) {
    h.qcell[nm - 1] = make_int4(zuv_md[nm] - 1, zuv_mu[nm] - 1, zuv_nd[nm] - 1, zuv_nu[nm] - 1);
    h.qlev[nm - 1] = (uint8_t)(iref_of[nm] - 1);
    h.qmap_u[nm - 1] = zuv_mu[nm] - 1;
    h.qmap_v[nm - 1] = zuv_nu[nm] - 1;
    h.flags[nm - 1] = (uint16_t)(F_ACT | (kcs[nm] == 1 ? F_KCS1 : 0));
    h.kcs_cmp[nm - 1] = kcs[nm];
    h.cmp_off[nm - 1] = (int32_t)(nm - 1);
    h.dense2cmp[nm - 1] = (int32_t)(nm - 1);
    if (kcs[nm] == 1) {
      h.n_kcs1++;
      h.area_total_kcs1 += (double)h.cell_area[nm - 1];
    }
  }
  h.qcuv.resize(ncuv);
  for (long ic = 1; ic <= ncuv; ic++) h.qcuv[ic - 1] = make_int2(cuv_uv1[ic] - 1, cuv_uv2[ic] - 1);
  // infiltration con (sfincs_infiltration.f90:8-606)
  P.infiltration = 0;
  if (P.precip && k.qinf > 0.0f) {
    P.infiltration = 1;
    h.qinf.assign(np, 0.0f);
    for (long i = 0; i < np; i++) {
      const float zz = P.subgrid ? h.zz_min[i] : h.zb[i];
      h.qinf[i] = zz > k.qinf_zmin ? k.qinf : 0.0f;
    }
  } else if (P.precip && !none(k.qinffile)) {  // c2d: a binary field in cell order, mm/h
    P.infiltration = 1;
    const auto r = read_binary<float>(h.dir + "/" + k.qinffile, (size_t)np);
    h.qinf.assign(np, 0.0f);
    for (long i = 0; i < np; i++) h.qinf[i] = r[(size_t)i] / 3600.0f / 1000.0f;
  }
  // restart file (sfincs_initial_conditions.F90:183-268): zs, q in the
  // reference's uv order (which is this mesh's), uvmean in boundary-face order
  RestartData rst;
  // the reference's uvmean also holds the lateral (Neumann) faces of its boundary list
  if (!h.neu.empty() && (!none(k.rstfile) || h.trstout < 1.0e9))
    throw std::runtime_error("restart files on quadtree meshes with Neumann cells (msk 6) are not supported");
  if (!none(k.rstfile)) {
    rst = read_restart(h.dir + "/" + k.rstfile);
    if (rst.type >= 1 && rst.type <= 6) {
      if ((long)rst.zs.size() != np) throw std::runtime_error("restart file: zs has the wrong length");
      if (!rst.q.empty() && (long)rst.q.size() != npuv + ncuv + 1)
        throw std::runtime_error("restart file: q has the wrong length");
      if (!rst.uvmean.empty() && (long)rst.uvmean.size() != (long)h.bfaces.size())
        throw std::runtime_error("restart file: uvmean has the wrong length");
    }
  }
  {  // infiltration models with state: parameters in cell order (compact storage)
    std::vector<int32_t> ident((size_t)np);
    for (long i = 0; i < np; i++) ident[(size_t)i] = (int32_t)i;
    load_infiltration_models(h, k, (size_t)np, ident);
    apply_restart_infiltration(h, rst, ident);
  }
  // initial state (sfincs_initial_conditions.F90:98-106, sfincs_subgrid.F90:907-962)
  // binary ini file: real*4 levels in cell order (read_zsini_file, sfincs_initial_conditions.F90:270-288)
  std::vector<float> inizs;
  if (!rst.zs.empty()) inizs = rst.zs;
  else if (!none(k.inifile)) inizs = read_binary<float>(h.dir + "/" + k.inifile, (size_t)np);
  h.zs.assign(np, 0.0f);
  for (long i = 0; i < np; i++) {
    const float base = P.subgrid ? h.zz_min[i] : h.zb[i];
    h.zs[i] = (float)std::max((double)base, inizs.empty() ? (double)P.zini : (double)inizs[(size_t)i]);
  }
  // fluxes of the uv points from the restart and the velocities they imply
  // (:110-173); combined points start at zero as in the reference
  if (!rst.q.empty()) {
    const size_t NQ = (size_t)(npuv + ncuv + 1);
    h.q0u.assign(NQ, 0.0f);
    h.uv0u.assign(NQ, 0.0f);
    const int L = P.nlev;
    for (long ip = 1; ip <= npuv; ip++) {
      const float q = rst.q[(size_t)ip - 1];
      h.q0u[(size_t)ip - 1] = q;
      const float zsuv = std::max(h.zs[uv_nm[ip] - 1], h.zs[uv_nmu[ip] - 1]);
      float huv;
      if (P.subgrid) {
        const float2 zr = h.sgz_u[(size_t)ip - 1];
        if (!(zsuv > zr.x + P.huthresh)) continue;
        if (zsuv > zr.y - 1.0e-4f) {
          huv = h.sgw_u[(size_t)ip - 1].x + zsuv;
        } else {
          const float dzuv = (zr.y - zr.x) / (float)(L - 1);
          const int iuv = std::min(std::max((int)((zsuv - zr.x) / dzuv) + 1, 1), L - 1);
          const float facint = (zsuv - (zr.x + (float)(iuv - 1) * dzuv)) / dzuv;
          const UvRec& r = h.rec_u[(size_t)(iuv - 1) * npuv + (size_t)ip - 1];
          huv = r.havg + r.dhavg * facint;
        }
        huv = std::max(huv, P.huthresh);
      } else {
        if (!(zsuv > h.zbmx_q[(size_t)ip - 1])) continue;
        huv = std::max(zsuv - zbuv[ip], P.huthresh);
      }
      h.uv0u[(size_t)ip - 1] = std::max(std::min(q / huv, 4.0f), -4.0f);
    }
  }
  if (!rst.uvmean.empty()) h.uvmean0 = rst.uvmean;
  h.zsmax.assign(np, -999.0f);
  if (P.wiggle) h.zs0 = h.zs;
  if (P.subgrid) {
    const int L = P.nlev;
    h.zvol.assign(np, 0.0);
    h.vneg.assign(np, 0);
    for (long i = 0; i < np; i++) {
      const double zs = h.zs[i];
      const double area = (double)h.cell_area[i];
      if (zs >= (double)h.zz_max[i]) {
        h.zvol[i] = (double)h.zz_volmax[i] + area * (zs - (double)std::max(h.zz_max[i], -20.0f));
      } else {
        const float* dep = &sg_dep[(size_t)i * L];
        int ivol = 1;
        for (int il = 2; il <= L; il++)
          if ((double)dep[il - 1] > zs) {
            ivol = il - 1;
            break;
          }
        const float dzvol = h.zz_volmax[i] / (float)(L - 1);
        const float facint =
            (float)((zs - (double)dep[ivol - 1]) / (double)std::max(dep[ivol] - dep[ivol - 1], 0.001f));
        h.zvol[i] = (double)((float)(ivol - 1) * dzvol + facint * dzvol);
      }
      h.vneg[i] = h.zvol[i] < 0.0 ? 1 : 0;
    }
  }
  read_meteo_series(h, k, rotation);
}

// find_quadtree_cell (sfincs_quadtree.F90:764-820): the finest level whose cell
// at the point is active; returns the 1-based cell index, 0 outside.
int quadtree_cell_index(const HostModel& h, double xd, double yd) {
  const float x = (float)xd, y = (float)yd;
  const float xt = h.cosrot * (x - h.x0) + h.sinrot * (y - h.y0);
  const float yt = -h.sinrot * (x - h.x0) + h.cosrot * (y - h.y0);
  for (int L = h.p.nref; L >= 1; L--) {
    const float dxr = h.p.dx / (float)(1 << (L - 1)), dyr = h.p.dy / (float)(1 << (L - 1));
    const int64_t n = (int64_t)(yt / dyr) + 1, m = (int64_t)(xt / dxr) + 1;
    if (n < 1 || m < 1) return 0;
    const int64_t key = qt_key(L, m, n);
    auto it = std::lower_bound(h.qt_key.begin(), h.qt_key.end(), key);
    if (it != h.qt_key.end() && *it == key) return h.qt_key_cell[it - h.qt_key.begin()] + 1;
  }
  return 0;
}

void load_quadtree(HostModel& h, const Keys& k) {
  QtBuilder b(h, k);
  b.mesh();
  b.neighbours();
  b.geometry();
  b.bed();
  b.boundaries();
  b.finish();
  // point sources (sfincs_discharges.f90:95-178): the finest active cell at
  // each point (find_quadtree_cell), compact indices
  if (!none(k.srcfile)) {
    auto path = [&](const std::string& f) { return h.dir + "/" + f; };
    auto xy = read_table(path(k.srcfile));
    auto tb = read_table(path(k.disfile));
    const int nsrc = (int)xy.size();
    for (auto& r : xy) {
      const int nm = quadtree_cell_index(h, r.at(0), r.at(1));
      if (nm <= 0) throw std::runtime_error("point source outside the active mesh");
      h.src_cell.push_back((int32_t)(nm - 1));
    }
    for (auto& r : tb) {
      if ((int)r.size() < nsrc + 1) throw std::runtime_error("dis file has fewer columns than src points");
      h.tsrc.push_back((float)r[0]);
      for (int is = 0; is < nsrc; is++) h.qsrc.push_back((float)r[is + 1]);
    }
    h.p.nsrc = nsrc;
    h.p.ntsrc = (int)h.tsrc.size();
  }
  // drainage structures: intake and outfall cells after the point sources
  if (!none(k.drnfile)) {
    auto path = [&](const std::string& f) { return h.dir + "/" + f; };
    for (const DrnLine& r : read_drainage(path(k.drnfile))) {
      const int ni = quadtree_cell_index(h, r.xs, r.ys), no = quadtree_cell_index(h, r.xo, r.yo);
      if (ni <= 0 || no <= 0) throw std::runtime_error("drainage point outside the active mesh");
      DrnDev d{};
      d.type = r.type;
      d.cin = ni - 1;
      d.cout = no - 1;
      for (int j = 0; j < 6; j++) d.p[j] = r.p[j];
      const float xsnk = h.z_xz[ni - 1], ysnk = h.z_yz[ni - 1], xsrc = h.z_xz[no - 1], ysrc = h.z_yz[no - 1];
      d.distance = std::sqrt((xsrc - xsnk) * (xsrc - xsnk) + (ysrc - ysnk) * (ysrc - ysnk));
      h.drn.push_back(d);
      h.src_cell.push_back((int32_t)(ni - 1));
      h.src_cell.push_back((int32_t)(no - 1));
    }
  }
  h.p.ndrn = (int)h.drn.size();
}

}  // namespace sfg
