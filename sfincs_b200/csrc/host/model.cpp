// Model loading (reference input files -> dense B200 layout), device
// residency and the CUDA-graph step runner.
#include "model.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <type_traits>
#include <stdexcept>

#include "inputs.h"

namespace sfg {

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

static bool is_none(const std::string& s) { return s.size() >= 4 && s.compare(0, 4, "none") == 0; }

void apply_restart_infiltration(HostModel& h, const RestartData& rst, const std::vector<int32_t>& store) {
  if (rst.type < 4 || rst.type > 6) return;  // flavours 4 cnb, 5 gai, 6 hor: the state overwrites the inputs
  if (h.p.inftype != rst.type - 1)
    throw std::runtime_error("restart file flavour " + std::to_string(rst.type) +
                             " carries the state of another infiltration method than the model's");
  for (int j = 0; j < (rst.type == 5 ? 2 : 1); j++) {
    if ((long long)rst.inf[j].size() != h.np) throw std::runtime_error("restart file: infiltration state has the wrong length");
    for (long long i = 0; i < h.np; i++) h.inf_st[j][(size_t)store[(size_t)i]] = rst.inf[j][(size_t)i];
  }
}

void load_infiltration_models(HostModel& h, const Keys& k, size_t nstore, const std::vector<int32_t>& store) {
  ScnDev& P = h.p;
  const size_t n = (size_t)h.np;
  if (P.store_cumprcp && P.precip) {
    h.cumprcp.assign(nstore, 0.0f);
    h.cuminf.assign(nstore, 0.0f);
  }
  if (P.inftype < 2) return;
  P.inf_last = store[n - 1];
  auto rd = [&](const std::string& f, const char* what) {
    if (is_none(f)) throw std::runtime_error(std::string("infiltration needs the ") + what + " file");
    return read_binary<float>(h.dir + "/" + f, n);
  };
  auto field = [&](std::vector<float>& dst, const std::vector<float>& src) {
    dst.assign(nstore, 0.0f);
    for (size_t i = 0; i < n; i++) dst[(size_t)store[i]] = src[i];
  };
  auto state = [&](int j, float v) { h.inf_st[j].assign(nstore, v); };
  if (P.inftype == 2) {  // cna: S in inches -> m (:249-279)
    auto r = rd(k.scsfile, "scs");
    for (auto& x : r) x = x * 0.0254f;
    field(h.inf_par[0], r);
  } else if (P.inftype == 3) {  // cnb: Smax, Se, recovery from ks in mm/h (:280-360, equation 4-36)
    auto smax = rd(k.smaxfile, "smax"), se = rd(k.sefffile, "seff"), ks = rd(k.ksfile, "ks");
    std::vector<float> kr(n);
    for (size_t i = 0; i < n; i++) kr[i] = std::sqrt(ks[i] / 25.4f) / 75.0f;
    field(h.inf_par[0], smax);
    field(h.inf_par[1], kr);
    field(h.inf_st[0], se);
    for (int j = 1; j <= 4; j++) state(j, 0.0f);
    h.inf_rain.assign(nstore, 0);
  } else if (P.inftype == 4) {  // gai (:361-505, equations 4-33 and 4-36)
    auto psi = rd(k.psifile, "psi"), sig = rd(k.sigmafile, "sigma"), ks = rd(k.ksfile, "ks");
    std::vector<float> kr(n), lu(n), ksm(n), head(n);
    for (size_t i = 0; i < n; i++) {
      kr[i] = std::sqrt(ks[i] / 25.4f) / 75.0f;
      lu[i] = 4.0f * std::sqrt(25.4f) * std::sqrt(ks[i]) / 1000.0f;
      head[i] = psi[i] / 1000.0f;
      ksm[i] = ks[i] / 1000.0f / 3600.0f;
    }
    field(h.inf_par[0], ksm);
    field(h.inf_par[1], sig);
    field(h.inf_par[2], lu);
    field(h.inf_par[3], kr);
    field(h.inf_par[4], head);
    field(h.inf_st[0], sig);  // sigma starts at its maximum
    state(1, 0.0f);
    state(2, 0.0f);
    state(3, 0.0f);
  } else if (P.inftype == 5) {  // hor: fc, f0 (mm/h), kd (1/h) (:506-590)
    auto fc = rd(k.fcfile, "fc"), f0 = rd(k.f0file, "f0"), kd = rd(k.kdfile, "kd");
    field(h.inf_par[0], fc);
    field(h.inf_par[1], f0);
    field(h.inf_par[2], kd);
    state(0, 0.0f);
  }
}

// The hu**(7/3) lookup table of h73table (fill_h73_tables, sfincs_data.f90:
// 858-881): x73(j, k) = hh**2 * hh**(1.0/3.0) at hh = 0.001 j 10**(k - 6),
// j = 1..1000, k = 1..10, in real*4 (10.0**(k - 6) for k < 6 as the reciprocal
// of the exact power), stored at (k - 1) * 1000 + j - 1.
static void fill_h73_table(std::vector<float>& x73) {
  x73.assign(10000, 0.0f);
  for (int k = 1; k <= 10; k++) {
    float p10 = 1.0f;
    for (int i = 0; i < std::abs(k - 6); i++) p10 = p10 * 10.0f;
    if (k < 6) p10 = 1.0f / p10;
    for (int j = 1; j <= 1000; j++) {
      const float hh = 0.001f * (float)j * p10;
      x73[(size_t)(k - 1) * 1000 + (j - 1)] = hh * hh * std::pow(hh, 1.0f / 3.0f);
    }
  }
}

// ============================================================================
// load_model
// ============================================================================
// Water-level boundary points and their time series (sfincs_boundaries.f90:8-213).
void read_boundary_series(HostModel& h, const Keys& k, bool water_level_bnd, std::vector<float>& xb,
                          std::vector<float>& yb, int& nbnd) {
  ScnDev& P = h.p;
  auto path = [&](const std::string& f) { return h.dir + "/" + f; };
  int ntbnd = 0;
  nbnd = 0;
  if (!is_none(k.bndfile)) {
    auto xy = read_table(path(k.bndfile));
    nbnd = (int)xy.size();
    for (auto& r : xy) {
      xb.push_back((float)r.at(0));
      yb.push_back((float)r.at(1));
    }
    if (!is_none(k.bzsfile)) {
      auto tb = read_table(path(k.bzsfile));
      ntbnd = (int)tb.size();
      h.zs_bnd.assign((size_t)ntbnd * nbnd, 0.0f);
      for (int it = 0; it < ntbnd; it++) {
        if ((int)tb[it].size() < nbnd + 1) throw std::runtime_error("bzs file has fewer columns than bnd points");
        h.t_bnd.push_back((float)tb[it][0]);
        for (int ib = 0; ib < nbnd; ib++) h.zs_bnd[(size_t)it * nbnd + ib] = (float)tb[it][ib + 1];
      }
    } else {
      ntbnd = 2;
      h.t_bnd = {k.t0, k.t1};
      h.zs_bnd.assign((size_t)2 * nbnd, 0.0f);
    }
    if (ntbnd < 1) throw std::runtime_error("empty boundary time series");
    if (h.t_bnd[0] > (k.t0 + 1.0f) || h.t_bnd[ntbnd - 1] < (k.t1 - 1.0f)) {
      if (h.t_bnd[0] > (k.t0 + 1.0f))
        h.t_bnd[0] = k.t0 - 1.0f;
      else
        h.t_bnd[ntbnd - 1] = k.t1 + 1.0f;
    }
  } else if (water_level_bnd) {
    nbnd = 1;
    xb = {0.0f};
    yb = {0.0f};
    ntbnd = 2;
    h.t_bnd = {k.t0, k.t1};
    h.zs_bnd = {0.0f, 0.0f};
  }
  P.nbnd = nbnd;
  P.ntbnd = ntbnd;
  // astronomic constituents of the boundary points, nodal-corrected at tref (sfincs_boundaries.f90:289-450)
  h.tide = TideHost{};
  if (!is_none(k.bcafile) && nbnd > 0) read_bca_file(path(k.bcafile), h.tref, nbnd, h.tide);
  P.ntide = h.tide.ncomp;
}

// Uniform wind and rain time series and the wind drag table (sfincs_meteo.f90:247-327).
void read_meteo_series(HostModel& h, const Keys& k, float rotation) {
  ScnDev& P = h.p;
  auto path = [&](const std::string& f) { return h.dir + "/" + f; };
  // gridded meteo with the enhancement factors (sfincs_meteo.f90:146-245, 330-380)
  if (!is_none(h.amufile)) {
    read_meteo_grid(path(h.amufile), h.tref, h.mgh[0], 0);
    read_meteo_grid(path(h.amvfile), h.tref, h.mgh[0], 1);
    if (h.factor_wind != 1.0f)
      for (int q = 0; q < 2; q++)
        for (auto& x : h.mgh[0].v[q]) x = h.factor_wind * x;
  }
  if (!is_none(h.ampfile)) {
    read_meteo_grid(path(h.ampfile), h.tref, h.mgh[1], 0);
    if (h.factor_pres != 1.0f)
      for (auto& x : h.mgh[1].v[0]) x = P.gapres - h.factor_pres * (P.gapres - x);
  }
  if (!is_none(h.amprfile)) {
    read_meteo_grid(path(h.amprfile), h.tref, h.mgh[2], 0);
    if (h.factor_prcp != 1.0f)
      for (auto& x : h.mgh[2].v[0]) x = h.factor_prcp * x;
  }
  if (!is_none(h.spwfile)) {  // spiderweb (sfincs_meteo.f90:35-98) with its factors (:330-412)
    SpwHost& w = h.spw;
    read_spw_file(path(h.spwfile), h.tref, h.use_spw_precip, w);
    h.spw_pabs.resize(w.pdrp.size());
    for (size_t i = 0; i < w.pdrp.size(); i++) h.spw_pabs[i] = P.gapres - w.pdrp[i];
    if (h.factor_wind != 1.0f) {
      for (auto& x : w.wu) x = h.factor_wind * x;
      for (auto& x : w.wv) x = h.factor_wind * x;
    }
    if (h.factor_pres != 1.0f)
      for (auto& x : h.spw_pabs) x = P.gapres - h.factor_pres * (P.gapres - x);
    if (w.precip && h.factor_prcp != 1.0f)
      for (auto& x : w.prcp) x = h.factor_prcp * x;
    if (h.factor_spw_size != 1.0f) w.radius = h.factor_spw_size * w.radius;
    P.spw.nt = w.nt;
    P.spw.nrows = w.nrows;
    P.spw.ncols = w.ncols;
    P.spw.precip = w.precip;
    P.spw.radius = w.radius;
    P.spw.drad = w.radius / (float)w.nrows;
    P.spw.dphi = 2.0f * P.pi / (float)w.ncols;
    P.spw.merge_frac = h.spw_merge_frac;
  }
  P.cosrot = std::cos(rotation);
  P.sinrot = std::sin(rotation);
  if (P.wind && !is_none(k.wndfile)) {
    auto tb = read_table(path(k.wndfile));
    for (auto& r : tb) {
      h.twnd.push_back((float)r.at(0));
      h.wmag.push_back((float)r.at(1));
      h.wdir.push_back(P.pi * (270.0f - (float)r.at(2)) / 180.0f - rotation);
    }
    P.ntwnd = (int)h.twnd.size();
    if (P.ntwnd < 2) throw std::runtime_error("wind time series needs at least two records");
  }
  if (P.precip && !is_none(k.prcpfile)) {
    auto tb = read_table(path(k.prcpfile));
    for (auto& r : tb) {
      h.tprcp.push_back((float)r.at(0));
      h.vprcp.push_back((float)r.at(1));
    }
    P.ntprcp = (int)h.tprcp.size();
    if (P.ntprcp < 1) throw std::runtime_error("empty precipitation time series");
  }
  {
    const float cd_wnd[3] = {0.0f, 28.0f, 50.0f}, cd_val[3] = {0.0010f, 0.0025f, 0.0015f};
    h.cdval.assign(1000, 0.0f);
    for (int iw = 1; iw <= 1000; iw++) {
      const float wnd = (float)iw * 0.1f;
      for (int icd = 1; icd <= 2; icd++) {
        h.cdval[iw - 1] = cd_val[icd - 1];
        if (wnd >= cd_wnd[icd - 1] && wnd < cd_wnd[icd]) {
          h.cdval[iw - 1] = cd_val[icd - 1] + (wnd - cd_wnd[icd - 1]) * (cd_val[icd] - cd_val[icd - 1]) /
                                                  (cd_wnd[icd] - cd_wnd[icd - 1]);
          break;
        } else if (wnd >= cd_wnd[2]) {
          h.cdval[iw - 1] = cd_val[2];
          break;
        }
      }
    }
  }
}

// Keywords of sfincs.inp with the reference's defaults and the values derived
// from them (sfincs_input.f90:50-745); scalar switches go straight into h.p.
Keys parse_keys(const InpFile& in, HostModel& h, bool bmi) {
  ScnDev& P = h.p;

  // ---- keywords and defaults (sfincs_input.f90:50-343) ----------------------
  const int mmax = in.integer("mmax", 0), nmax = in.integer("nmax", 0);
  const float dx = in.real("dx", 0.0f), dy = in.real("dy", 0.0f);
  const float x0 = in.real("x0", 0.0f), y0 = in.real("y0", 0.0f);
  float rotation = in.real("rotation", 0.0f);
  std::string tref = in.str("tref", "none"), tstart = in.str("tstart", "20000101 000000"),
              tstop = in.str("tstop", "20000101 000000");
  float tspinup = in.real("tspinup", 0.0f);
  const float dtmaxout = in.real("dtmaxout", 9999999.0f);
  P.alfa = in.real("alpha", 0.50f);
  P.theta = in.real("theta", 1.0f);
  const float hmin_cfl = in.real("hmin_cfl", 0.1f);
  const float manning = in.real("manning", 0.04f), manning_land = in.real("manning_land", -999.0f),
              manning_sea = in.real("manning_sea", -999.0f), rghlevland = in.real("rgh_lev_land", 0.0f);
  P.zini = in.real("zsini", 0.0f);
  float qinf = in.real("qinf", 0.0f);
  float dtmax = in.real("dtmax", 60.0f);
  P.huthresh = in.real("huthresh", 0.05f);
  P.huvmin = in.real("huvmin", 0.0f);
  P.rhoa = in.real("rhoa", 1.25f);
  P.rhow = in.real("rhow", 1024.0f);
  const std::string inputtype = in.str("inputformat", "bin");
  const int bndtype = in.integer("bndtype", 1);
  const int iadvection = in.integer("advection", 1);
  const float latitude = in.real("latitude", 0.0f);
  P.advlim = in.real("advlim", 1.0f);
  P.slopelim = in.real("slopelim", 9999.9f);
  const float qinf_zmin = in.real("qinf_zmin", 0.0f);
  P.btfilter = in.real("btfilter", 60.0f);
  const int igeo = in.integer("crsgeo", 0);
  bool coriolis = in.logical("coriolis", true);
  const float nuviscdim = in.real("nuvisc", 0.01f);
  const bool viscosity = in.logical("viscosity", false);
  const std::string advstr = in.str("advection_scheme", "upw1");
  P.btrelax = in.real("btrelax", 3600.0f);
  const bool wiggle = in.logical("wiggle_suppression", true);
  P.wiggle_factor = in.real("wiggle_factor", 0.1f);
  P.wiggle_threshold = in.real("wiggle_threshold", 0.1f);
  P.uvlim = in.real("uvlim", 10.0f);
  const float uvmax = in.real("uvmax", 1000.0f);
  const bool friction2d = in.logical("friction2d", true);
  const bool advection_mask = in.logical("advection_mask", true);
  P.nuviscfac = in.real("nuviscfac", 100.0f);
  P.h73table = in.logical("h73table", false) ? 1 : 0;
  if (P.h73table) fill_h73_table(h.x73);
  const std::string qtrfile = in.str("qtrfile", "none"), depfile = in.str("depfile", "none"),
                    inifile = in.str("inifile", "none"), rstfile = in.str("rstfile", "none"),
                    mskfile = in.str("mskfile", "none"), indexfile = in.str("indexfile", "none"),
                    sbgfile = in.str("sbgfile", "none"), manningfile = in.str("manningfile", "none"),
                    bndfile = in.str("bndfile", "none"), bzsfile = in.str("bzsfile", "none"),
                    srcfile = in.str("srcfile", "none"), disfile = in.str("disfile", "none"),
                    wndfile = in.str("wndfile", "none"), qinffile = in.str("qinffile", "none");
  std::string prcpfile = in.str("prcfile", "none");
  if (is_none(prcpfile)) prcpfile = in.str("precipfile", "none");
  // Inputs outside this core's path: refuse loudly instead of silently ignoring physics.
  for (const char* k : {"bzifile", "volfile", "netbndbzsbzifile", "netsrcdisfile",
                        "netamuamvfile", "netamprfile", "netampfile", "netspwfile", "infiltration_file",
                        "wavemaker_wvmfile", "wvmfile"}) {
    if (!is_none(in.str(k, "none"))) throw std::runtime_error(std::string("input '") + k + "' is not supported by this core");
  }
  for (const char* k : {"snapwave", "nonh", "bathtub", "vegetation"})
    if (in.logical(k, false) || in.integer(k, 0) != 0)
      throw std::runtime_error(std::string("process '") + k + "' is not supported by this core");
  // A netCDF inifile goes through the reference's quadtree netCDF reader
  // (sfincs_initial_conditions.F90:61-78); the binary form is read below.
  if (!is_none(inifile) && inifile.size() >= 2 && inifile.compare(inifile.size() - 2, 2, "nc") == 0)
    throw std::runtime_error("netCDF inifile is not supported by this core (use the binary real*4 form)");
  // geographic grids (crsgeo, sfincs_input.f90:399-421): regular grids; the
  // options whose geographic arithmetic this core does not carry are refused
  if (igeo != 0) {
    if (!is_none(qtrfile)) throw std::runtime_error("geographic quadtree meshes (crsgeo=1 with qtrfile) are not supported");
    for (const char* k : {"spwfile", "weirfile", "drnfile", "crsfile"})
      if (!is_none(in.str(k, "none")))
        throw std::runtime_error(std::string("input '") + k + "' on a geographic grid (crsgeo=1) is not supported");
  }
  P.geo = igeo != 0 ? 1 : 0;
  if (inputtype != "bin") throw std::runtime_error("only inputformat = bin is supported");
  if (bndtype != 1) throw std::runtime_error("only bndtype = 1 is supported");
  const bool quadtree = !is_none(qtrfile);
  const std::string thdfile = in.str("thdfile", "none"), weirfile = in.str("weirfile", "none"),
                    drnfile = in.str("drnfile", "none");
  P.structure_relax = in.real("structure_relax", 10.0f);
  if (!quadtree && (nmax <= 0 || mmax <= 0)) throw std::runtime_error("nmax/mmax missing in sfincs.inp");

  // ---- derived (sfincs_input.f90:347-745) ------------------------------------
  if (is_none(tref)) tref = tstart;
  const float t0 = (float)(seconds_between(tref, tstart) * 1.0);
  const float t1 = (float)(seconds_between(tref, tstop) * 1.0);
  {  // restart output times (sfincs_input.f90:61-66, 441-444; sfincs_output.f90:39-56)
    float t0out = in.real("t0out", -999.0f);
    const float dtrstout = in.real("dtrstout", 0.0f), trst = in.real("trstout", -999.0f);
    if (t0out < -900.0f) t0out = t0;
    t0out = std::max(t0out, t0);
    h.tref = tref;
    h.dtrstout = dtrstout;
    h.trstout = dtrstout > 1.0e-6f ? (double)(t0out + dtrstout) : (trst > 1.0e-6f ? (double)trst : 1.0e9);
    // map / his / max output (sfincs_input.f90:61-87, 274-294, 341-343, 441-447, 532-535)
    OutputSpec& o = h.out;
    float t1out = in.real("t1out", -999.0f);
    if (t1out < -900.0f) t1out = t1;
    o.t0out = t0out;
    o.t1out = t1out;
    float dtmapout = in.real("dtout", 0.0f);
    if (dtmapout == 0.0f) dtmapout = in.real("dtmapout", 0.0f);
    o.dtmapout = dtmapout;
    o.dtmaxout = dtmaxout;
    o.dthisout = in.real("dthisout", 600.0f);
    const std::string otype = in.str("outputformat", "net");
    o.map_type = in.str("outputtype_map", "nil");
    o.his_type = in.str("outputtype_his", "nil");
    if (o.map_type == "nil" || o.his_type == "nil") o.map_type = o.his_type = otype;
    if (o.map_type != "net" && o.map_type != "bin" && o.map_type != "asc")
      throw std::runtime_error("outputformat '" + o.map_type + "' is not supported (net, bin or asc)");
    if (o.map_type == "asc" && dtmapout > 1.0e-6f)
      throw std::runtime_error("ASCII map output (outputformat = asc) is not supported; use net or bin");
    o.store_velocity = in.integer("storevel", 0) == 1;
    o.store_hsubgrid = in.integer("storehsubgrid", 0) == 1;
    o.store_zvolume = in.integer("storezvolume", 0) == 1;
    o.epsg = in.integer("epsg", 0);
    o.epsg_code = in.str("epsg_code", std::to_string(o.epsg));
    if (in.logical("storehmean", false)) throw std::runtime_error("storehmean (subgrid mean depth output) is not supported");
    if (in.integer("storemeteo", 0) == 1) throw std::runtime_error("storemeteo (meteo map output) is not supported");
    if (in.logical("debug", false)) throw std::runtime_error("debug output (every step) is not supported");
    o.crsfile = in.str("crsfile", "none");
    o.rugdepth = in.real("rugdepth", 0.05f);
    for (const auto& kv : in.all()) o.inp.push_back(kv);
  }
  tspinup = t0 + tspinup;
  P.g = 9.81f;
  P.pi = 3.14159f;
  qinf = qinf / (float)(3600 * 1000);
  rotation = rotation * P.pi / 180.0f;
  const float cosrot = std::cos(rotation), sinrot = std::sin(rotation);
  if (!P.geo) {  // projected: Coriolis from the latitude, off near the equator (geographic: per cell)
    P.fcorio = 2.0f * 7.2921e-05f * std::sin(latitude * P.pi / 180.0f);
    if (latitude < 0.01f && latitude > -0.01f) coriolis = false;
  }
  P.coriolis = coriolis;
  P.store_zsmax = dtmaxout > 0.0f;
  h.store_vmax = in.integer("storevelmax", 0) == 1 && dtmaxout > 0.0f;
  h.store_qmax = in.integer("storefluxmax", 0) == 1 && dtmaxout > 0.0f;
  h.store_twet = in.integer("storetwet", 0) == 1;
  P.store_vmax = h.store_vmax;
  P.store_qmax = h.store_qmax;
  P.store_twet = h.store_twet;
  P.store_tzsmax = in.integer("storetzsmax", 0) == 1 && P.store_zsmax;
  P.twet_threshold = in.real("twet_threshold", 0.01f);
  P.subgrid = !is_none(sbgfile);
  P.advection = iadvection > 0;
  P.adv_scheme = 1;
  if (P.advection && advstr == "original") P.adv_scheme = 0;
  P.thetasmooth = P.theta < 0.9999f;
  P.viscosity = viscosity;
  P.friction2d = friction2d;
  P.wiggle = wiggle;
  // meteo processes (sfincs_domain.f90:95-125): wind from a time series or
  // the amu / amv grids, pressure from the amp grid, rain from a time series or
  // the ampr grid; a quantity from both a grid and a time series is refused
  // (the reference lets the series overwrite the field and counts the
  // cumulative rain of both)
  {
    const std::string amu = in.str("amufile", "none"), amv = in.str("amvfile", "none"),
                      amp = in.str("ampfile", "none"), ampr = in.str("amprfile", "none");
    if (!is_none(amu) && is_none(amv)) throw std::runtime_error("amufile needs an amvfile");
    if (!is_none(amu) && !is_none(wndfile)) throw std::runtime_error("wind from both amufile and wndfile");
    if (!is_none(ampr) && !is_none(prcpfile)) throw std::runtime_error("rain from both amprfile and prcfile");
    if (in.real("waveage", -999.0f) > 0.0f) throw std::runtime_error("waveage (wave-age wind drag) is not supported");
    if (in.integer("radstr", 0) == 1) throw std::runtime_error("radstr is not supported");
    // spiderweb: a cyclone's polar wind / pressure / rain merged over the grids
    // (sfincs_meteo.f90:35-98, 450-800); its options that need tables or
    // projections outside this core are refused
    const std::string spw = in.str("spwfile", "none");
    const bool use_spw_precip = in.integer("usespwprecip", 1) != 0;
    bool spw_precip = false;
    if (!is_none(spw)) {
      if (!is_none(wndfile)) throw std::runtime_error("wind from both spwfile and wndfile");
      if (in.str("utmzone", "nil") != "nil") throw std::runtime_error("utmzone (spiderweb reprojection) is not supported");
      if (!is_none(in.str("z0lfile", "none")))
        throw std::runtime_error("z0lfile (wind reduction over land) is not supported");
      // n_quantity decides whether the web brings rain (read_meteo_data, :83-93)
      std::ifstream fs(h.dir + "/" + spw);
      for (std::string l; std::getline(fs, l) && l.compare(0, 4, "TIME") != 0;) {
        const size_t e = l.find('=');
        if (e == std::string::npos) continue;
        std::string k = l.substr(0, e);
        k.erase(0, k.find_first_not_of(" \t"));
        k.erase(k.find_last_not_of(" \t") + 1);
        if (k == "n_quantity" || k == "N_quantity") spw_precip = std::atoi(l.substr(e + 1).c_str()) == 4 && use_spw_precip;
      }
      if (spw_precip && !is_none(prcpfile)) throw std::runtime_error("rain from both spwfile and prcfile");
    }
    P.wind = !is_none(wndfile) || !is_none(amu) || !is_none(spw);
    P.wind_field = !is_none(amu) || !is_none(spw);
    P.patmos = (!is_none(amp) || !is_none(spw)) && in.integer("baro", 1) == 1;
    P.precip = !is_none(prcpfile) || !is_none(ampr) || spw_precip;
    P.prcp_field = !is_none(ampr) || spw_precip;
    P.meteo3d = !is_none(amu) || !is_none(amp) || !is_none(ampr) || !is_none(spw);
    h.spwfile = spw;
    h.use_spw_precip = use_spw_precip;
    h.spw_merge_frac = in.real("spwmergefrac", 0.5f);
    h.factor_spw_size = in.real("factor_spw_size", 1.0f);
    P.spinup_meteo = in.integer("spinup_meteo", 0) != 0;
    P.ampr_block = in.integer("amprblock", 1) != 0;
    P.dtwnd = in.real("dtwnd", 1800.0f);
    P.gapres = in.real("gapres", 101200.0f);
    P.pavbnd = in.real("pavbnd", 0.0f);
    h.amufile = amu;
    h.amvfile = amv;
    h.ampfile = P.patmos ? amp : std::string("none");
    h.amprfile = ampr;
    h.factor_wind = in.real("factor_wind", 1.0f);
    h.factor_pres = in.real("factor_pres", 1.0f);
    h.factor_prcp = in.real("factor_prcp", 1.0f);
  }
  P.use_qext = bmi;
  P.t0 = t0;
  P.t1 = t1;
  P.tspinup = tspinup;
  h.t0 = t0;
  h.t1 = t1;
  if (P.subgrid) P.huthresh = 0.0f;  // sfincs_subgrid.F90:40 (netCDF tables)
  Keys k;
  k.mmax = mmax; k.nmax = nmax; k.dx = dx; k.dy = dy; k.x0 = x0; k.y0 = y0; k.rotation = rotation;
  k.cosrot = cosrot; k.sinrot = sinrot; k.t0 = t0; k.t1 = t1; k.hmin_cfl = hmin_cfl; k.dtmax = dtmax;
  k.uvmax = uvmax; k.nuviscdim = nuviscdim; k.viscosity = viscosity; k.manning = manning;
  k.manning_land = manning_land; k.manning_sea = manning_sea; k.rghlevland = rghlevland; k.qinf = qinf;
  k.qinf_zmin = qinf_zmin; k.advection_mask = advection_mask; k.qtrfile = qtrfile; k.depfile = depfile;
  k.mskfile = mskfile; k.indexfile = indexfile; k.sbgfile = sbgfile; k.manningfile = manningfile;
  k.bndfile = bndfile; k.bzsfile = bzsfile; k.srcfile = srcfile; k.disfile = disfile; k.wndfile = wndfile;
  k.qinffile = qinffile; k.prcpfile = prcpfile; k.quadtree = quadtree; k.thdfile = thdfile; k.weirfile = weirfile; k.drnfile = drnfile; k.rstfile = rstfile;
  k.inifile = inifile;
  k.bdrfile = in.str("bdrfile", "none");
  // astronomic constituents apply when use_bcafile (default on) and a bca file is given (sfincs_input.f90:199, 231)
  k.bcafile = in.logical("use_bcafile", true) ? in.str("bcafile", "none") : std::string("none");
  k.scsfile = in.str("scsfile", "none");
  k.smaxfile = in.str("smaxfile", "none");
  k.sefffile = in.str("sefffile", "none");
  k.ksfile = in.str("ksfile", "none");
  k.psifile = in.str("psifile", "none");
  k.sigmafile = in.str("sigmafile", "none");
  k.f0file = in.str("f0file", "none");
  k.fcfile = in.str("fcfile", "none");
  k.kdfile = in.str("kdfile", "none");
  // infiltration type (sfincs_infiltration.f90:61-145): con / c2d first, then
  // the models with state; all of it only with rain
  P.sfacinf = in.real("sfacinf", 0.2f);
  P.horton_kr_kd = in.real("horton_kr_kd", 10.0f);
  P.store_cumprcp = in.integer("storecumprcp", 0) == 1;
  P.inftype = 0;
  if (P.precip) {
    if (qinf > 0.0f || !is_none(qinffile)) P.inftype = 1;
    else if (!is_none(k.scsfile)) P.inftype = 2;
    else if (!is_none(k.sefffile)) P.inftype = 3;
    else if (!is_none(k.psifile)) P.inftype = 4;
    else if (!is_none(k.f0file)) P.inftype = 5;
  }
  if (P.inftype == 2 || P.inftype == 3) P.store_cumprcp = 1;  // the curve-number methods need the sums
  return k;
}

// ---- thin dams and weirs (sfincs_structures.f90:38-495) --------------------------
// A .thd / .weir file holds polylines, each as a name line, an "nrows ncols"
// line and nrows lines of x y followed by npars values per point (blank lines
// skipped, commas accepted as separators, as list-directed input does).
std::vector<std::vector<PolyRow>> read_polylines(const std::string& file, int npars, std::vector<std::string>* names) {
  FILE* fp = std::fopen(file.c_str(), "r");
  if (!fp) throw std::runtime_error("cannot open polyline file " + file);
  std::vector<std::string> lines;
  char buf[4096];
  while (std::fgets(buf, sizeof buf, fp)) {
    std::string l(buf);
    for (char& ch : l)
      if (ch == ',' || ch == '\t' || ch == '\r' || ch == '\n') ch = ' ';
    if (l.find_first_not_of(' ') != std::string::npos) lines.push_back(l);
  }
  std::fclose(fp);
  std::vector<std::vector<PolyRow>> out;
  size_t i = 0;
  while (i + 1 < lines.size()) {
    if (names) {  // the name: the line's first item, a quoted string whole (list-directed read)
      const std::string& l = lines[i];
      const size_t a = l.find_first_not_of(' ');
      std::string nm;
      if (l[a] == '\'' || l[a] == '"') {
        const size_t b = l.find(l[a], a + 1);
        nm = l.substr(a + 1, (b == std::string::npos ? l.size() : b) - a - 1);
      } else {
        std::istringstream(l) >> nm;
      }
      names->push_back(nm);
    }
    i++;  // name line
    int nrows = 0, ncols = 0;
    if (std::sscanf(lines[i++].c_str(), "%d %d", &nrows, &ncols) != 2 || nrows < 0)
      throw std::runtime_error("polyline file " + file + ": bad block header");
    std::vector<PolyRow> pl;
    for (int r = 0; r < nrows; r++) {
      PolyRow row{};
      if (i >= lines.size() ||
          std::sscanf(lines[i++].c_str(), "%f %f %f %f", &row.x, &row.y, &row.p[0], &row.p[1]) < 2 + npars)
        throw std::runtime_error("polyline file " + file + ": truncated polyline");
      pl.push_back(row);
    }
    out.push_back(std::move(pl));
  }
  return out;
}

float crossing_sign(float xnm, float ynm, float xnmu, float ynmu, float xa, float ya, float xb, float yb, float pi) {
  const float phiuv = std::atan2(ynmu - ynm, xnmu - xnm);
  const float phic = std::atan2(yb - ya, xb - xa);
  float dphi = phiuv - phic;
  if (dphi < 0.0f) dphi = dphi + 2.0f * pi;
  if (dphi > 2.0f * pi) dphi = dphi - 2.0f * pi;
  return dphi <= pi ? 1.0f : -1.0f;
}

// Drainage structures file (sfincs_discharges.f90:203-256): one line each,
// "x_intake y_intake x_outfall y_outfall type params...", with 1 parameter for
// types 1-3 and 6 for the gates (4, 5).
std::vector<DrnLine> read_drainage(const std::string& file) {
  FILE* fp = std::fopen(file.c_str(), "r");
  if (!fp) throw std::runtime_error("cannot open drainage file " + file);
  std::vector<DrnLine> out;
  char buf[4096];
  while (std::fgets(buf, sizeof buf, fp)) {
    std::string l(buf);
    for (char& ch : l)
      if (ch == ',' || ch == '\t' || ch == '\r' || ch == '\n') ch = ' ';
    if (l.find_first_not_of(' ') == std::string::npos) continue;
    DrnLine d{};
    const int got = std::sscanf(l.c_str(), "%f %f %f %f %d %f %f %f %f %f %f", &d.xs, &d.ys, &d.xo, &d.yo, &d.type,
                                &d.p[0], &d.p[1], &d.p[2], &d.p[3], &d.p[4], &d.p[5]);
    const int npars = (d.type >= 1 && d.type <= 3) ? 1 : ((d.type == 4 || d.type == 5) ? 6 : 0);
    if (got < 5 || npars == 0) {
      std::fclose(fp);
      throw std::runtime_error("drainage type not recognized in " + file);
    }
    if (got < 5 + npars) {
      std::fclose(fp);
      throw std::runtime_error("drainage type " + std::to_string(d.type) + " requires " + std::to_string(npars) +
                               " parameters");
    }
    for (int k = npars; k < 6; k++) d.p[k] = 0.0f;
    out.push_back(d);
  }
  std::fclose(fp);
  return out;
}

// Length of the projection of the segment a-b onto the line segment 1-2,
// each end clamped to the segment (third_party_open/utils/geometry.f90:215-297).
float projected_length(float x0a, float y0a, float x0b, float y0b, float x1, float y1, float x2, float y2) {
  const float aa = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
  auto along = [&](float px, float py, float& b) {
    b = std::fabs((x2 - x1) * (y1 - py) - (x1 - px) * (y2 - y1)) / std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    const float c1 = std::sqrt((px - x1) * (px - x1) + (py - y1) * (py - y1));
    const float c2 = std::sqrt((px - x2) * (px - x2) + (py - y2) * (py - y2));
    const float a1 = std::sqrt(std::max(c1 * c1 - b * b, 0.0f)), a2 = std::sqrt(std::max(c2 * c2 - b * b, 0.0f));
    if (a1 > aa || a2 > aa) return a1 < a2 ? 0.0f : 1.0f;
    return a1 / aa;
  };
  float b1 = 0.0f, b2 = 0.0f;
  const float p1 = along(x0a, y0a, b1), p2 = along(x0b, y0b, b2);
  return (b1 < 999999.0f && b2 < 999999.0f) ? aa * std::fabs(p2 - p1) : 0.0f;
}

// Side of c relative to the line a -> b, with the 1e-6 dead band of the
// reference's geometry helper (FP32 throughout, like the reference's real*4).
static int side_of(float ax, float ay, float bx, float by, float cx, float cy) {
  const float val = (by - ay) * (cx - bx) - (bx - ax) * (cy - by);
  return val < -1.0e-6f ? -1 : (val > 1.0e-6f ? 1 : 0);
}

// Segments p1-p2 and q1-q2 cross when each separates the other's end points
// (a touching or collinear end point counts as on neither side).
bool segments_cross(float p1x, float p1y, float p2x, float p2y, float q1x, float q1y, float q2x, float q2y) {
  return side_of(p1x, p1y, p2x, p2y, q1x, q1y) != side_of(p1x, p1y, p2x, p2y, q2x, q2y) &&
         side_of(q1x, q1y, q2x, q2y, p1x, p1y) != side_of(q1x, q1y, q2x, q2y, p2x, p2y);
}

// ---- binary restart files (sfincs_initial_conditions.F90:183-268) -------------------
// Fortran unformatted sequential records, each framed by its byte length:
// the flavour (int32), zs (float32[np]), and for flavours 1, 2, 4-6 the fluxes
// q (float32[npuv + ncuv + 1], reference face order) and the boundary mean
// fluxes uvmean (float32[nkcuv2]).
RestartData read_restart(const std::string& file) {
  FILE* fp = std::fopen(file.c_str(), "rb");
  if (!fp) throw std::runtime_error("cannot open restart file " + file);
  std::vector<std::vector<char>> rec;
  for (;;) {
    int32_t len = 0, tail = 0;
    if (std::fread(&len, 4, 1, fp) != 1) break;
    if (len < 0) throw std::runtime_error("restart file " + file + ": bad record");
    std::vector<char> r((size_t)len);
    if ((len > 0 && std::fread(r.data(), 1, (size_t)len, fp) != (size_t)len) || std::fread(&tail, 4, 1, fp) != 1 ||
        tail != len) {
      std::fclose(fp);
      throw std::runtime_error("restart file " + file + ": truncated record");
    }
    rec.push_back(std::move(r));
  }
  std::fclose(fp);
  RestartData d;
  if (rec.empty() || rec[0].size() != 4) throw std::runtime_error("restart file " + file + ": no flavour record");
  std::memcpy(&d.type, rec[0].data(), 4);
  auto floats = [&](size_t i) {
    if (i >= rec.size() || rec[i].size() % 4) throw std::runtime_error("restart file " + file + ": missing record");
    std::vector<float> v(rec[i].size() / 4);
    std::memcpy(v.data(), rec[i].data(), rec[i].size());
    return v;
  };
  if (d.type < 1 || d.type > 6) return d;  // the reference skips an unknown flavour with a warning
  d.zs = floats(1);
  if (d.type != 3) {  // q and uvmean in every flavour but 3 (sfincs_initial_conditions.F90:227-235)
    d.q = floats(2);
    d.uvmean = floats(3);
  }
  if (d.type == 4 || d.type == 6) d.inf[0] = floats(4);  // scs_Se / rain_T1 (:237-258)
  if (d.type == 5) {                                    // GA_sigma, GA_F
    d.inf[0] = floats(4);
    d.inf[1] = floats(5);
  }
  return d;
}

std::unique_ptr<HostModel> load_model(const std::string& dir, bool bmi) {
  auto H = std::make_unique<HostModel>();
  HostModel& h = *H;
  ScnDev& P = h.p;
  h.dir = dir;
  auto path = [&](const std::string& f) { return dir + "/" + f; };
  InpFile in(path("sfincs.inp"));
  const Keys K = parse_keys(in, h, bmi);
  // bounded wait of the staged kernels; SFG_TEST_WAIT_ROUNDS lowers it so a
  // test can make the wait give up (the fault path) without a fault on the GPU
  P.wait_limit = 1 << 22;
  if (const char* w = std::getenv("SFG_TEST_WAIT_ROUNDS")) P.wait_limit = std::max(0, std::atoi(w));
  if (K.quadtree) {
    load_quadtree(h, K);
    read_obs_points(h);
    return H;
  }
  const int mmax = K.mmax, nmax = K.nmax;
  const float dx = K.dx, dy = K.dy, x0 = K.x0, y0 = K.y0, rotation = K.rotation, cosrot = K.cosrot,
              sinrot = K.sinrot, t0 = K.t0, t1 = K.t1, hmin_cfl = K.hmin_cfl, dtmax = K.dtmax, uvmax = K.uvmax,
              nuviscdim = K.nuviscdim, manning = K.manning, manning_land = K.manning_land,
              manning_sea = K.manning_sea, rghlevland = K.rghlevland, qinf = K.qinf, qinf_zmin = K.qinf_zmin;
  const bool viscosity = K.viscosity, advection_mask = K.advection_mask;
  const std::string &depfile = K.depfile, &mskfile = K.mskfile, &indexfile = K.indexfile, &sbgfile = K.sbgfile,
                    &manningfile = K.manningfile, &bndfile = K.bndfile, &bzsfile = K.bzsfile,
                    &srcfile = K.srcfile, &disfile = K.disfile, &wndfile = K.wndfile, &qinffile = K.qinffile,
                    &prcpfile = K.prcpfile;

  // ---- mesh: index + mask files (sfincs_domain.f90:250-482) -------------------
  const long long n_idx = read_binary<int32_t>(path(indexfile), 1)[0];
  auto idx = read_binary<int32_t>(path(indexfile), (size_t)n_idx, 4);
  auto msk_idx = read_binary<int8_t>(path(mskfile), (size_t)n_idx);
  P.nmax = nmax;
  P.mmax = mmax;
  const int ld = ((nmax + 1 + kGhostPad + 1) + 31) / 32 * 32;
  P.ld = ld;
  P.nalloc = (int64_t)(mmax + 2) * ld;
  P.dx = dx;
  P.dy = dy;
  const size_t NA = (size_t)P.nalloc;
  auto OFF = [&](int n, int m) -> int64_t { return (int64_t)m * ld + kGhostPad + n; };
  std::vector<int8_t> kcs(NA, 0);
  std::vector<int32_t> cmp_of(NA, -1);  // dense -> compact index (0-based)
  for (long long i = 0; i < n_idx; i++) {
    if (msk_idx[i] <= 0) continue;
    const int m = (idx[i] - 1) / nmax + 1;
    const int n = idx[i] - (m - 1) * nmax;
    if (m < 1 || m > mmax || n < 1 || n > nmax) throw std::runtime_error("index file entry outside the grid");
    const int64_t c = OFF(n, m);
    kcs[c] = msk_idx[i];
    cmp_of[c] = (int32_t)h.cmp_off.size();
    h.cmp_off.push_back((int32_t)c);
    h.z_n.push_back(n);
    h.z_m.push_back(m);
  }
  h.np = (long long)h.cmp_off.size();
  for (int8_t k : kcs)
    if (k == 4) throw std::runtime_error("msk value 4 (wave makers) is not supported");
  auto act = [&](int n, int m) { return n >= 1 && n <= nmax && m >= 1 && m <= mmax && kcs[OFF(n, m)] > 0; };

  // ---- geometry (sfincs_domain.f90:1369-1541, projected, one level) -----------
  P.dxinv = 1.0f / dx;
  P.dyinv = 1.0f / dy;
  P.dx2inv = P.dxinv * P.dxinv;
  P.dy2inv = P.dyinv * P.dyinv;
  P.area = dx * dy;
  P.nref = 1;
  float dxymin = 1.0e6f;
  dxymin = std::min(dxymin, dx);
  dxymin = std::min(dxymin, dy);
  P.dtmax = std::min(dtmax, P.alfa * dxymin / (std::sqrt(9.81f * hmin_cfl)));
  P.dtmin = P.alfa * dxymin / (1.25f * std::fabs(uvmax));
  P.nuvisc = viscosity ? std::max(nuviscdim * std::min(dx, dy), 0.0f) : 0.0f;
  h.z_xz.resize(h.np);
  h.z_yz.resize(h.np);
  for (long long i = 0; i < h.np; i++) {
    const float n = (float)h.z_n[i], m = (float)h.z_m[i];
    h.z_xz[i] = x0 + cosrot * (1.0f * (m - 0.5f)) * dx - sinrot * (1.0f * (n - 0.5f)) * dy;
    h.z_yz[i] = y0 + sinrot * (1.0f * (m - 0.5f)) * dx + cosrot * (1.0f * (n - 0.5f)) * dy;
  }
  if (P.geo) {  // geographic: dx, dy in degrees (sfincs_domain.f90:1403-1473, 1549-1559)
    P.geo_dyrm = 111111.1f * dy;
    P.dyinv = 1.0f / P.geo_dyrm;
    P.dy2inv = P.dyinv * P.dyinv;
    P.dtmax = dtmax;  // no limit from the spacing, and no dtmin, on geographic grids
    P.dtmin = 0.0f;
    P.nuvisc = viscosity ? std::max(nuviscdim * std::min(dx, dy) / 0.00001f, 0.0f) : 0.0f;
    h.geo_dxm.assign(NA, 0.0f);
    h.geo_dxminv.assign(NA, 0.0f);
    h.geo_area.assign(NA, 0.0f);
    if (P.coriolis) h.geo_fcor.assign(NA, 0.0f);
    for (long long i = 0; i < h.np; i++) {
      const int64_t c = h.cmp_off[i];
      const float cl = std::cos(h.z_yz[i] * P.pi / 180.0f);
      h.geo_dxm[c] = dx * 111111.1f * cl;
      h.geo_dxminv[c] = 1.0f / (dx * 111111.1f * cl);
      h.geo_area[c] = h.geo_dxm[c] * P.geo_dyrm;
      if (P.coriolis) h.geo_fcor[c] = 2.0f * 7.2921e-05f * std::sin(h.z_yz[i] * P.pi / 180.0f);
    }
  }

  // ---- faces and their reference order (sfincs_domain.f90:727-1003) ----------
  // kcu/kcv: kcuv of the u/v face owned by each dense cell (0 where no face).
  std::vector<int8_t> kcu(NA, 0), kcv(NA, 0);
  std::vector<int64_t> face_off;  // compact face ip-1 -> dense offset
  std::vector<int8_t> face_dir;
  auto kcuv_of = [&](int a, int b) -> int8_t {  // sfincs_domain.f90:1833-1884
    if (a > 1 && b > 1) return 0;
    if (a * b == 0) return 0;
    if ((a == 1 && b == 2) || (a == 2 && b == 1)) return 2;
    if ((a == 1 && b == 3) || (a == 3 && b == 1)) return 2;
    if ((a == 1 && b == 5) || (a == 5 && b == 1)) return 2;
    if ((a == 1 && b == 6) || (a == 6 && b == 1)) return 6;
    return 1;
  };
  for (long long i = 0; i < h.np; i++) {
    const int n = h.z_n[i], m = h.z_m[i];
    const int64_t c = OFF(n, m);
    if (act(n, m + 1)) {
      face_off.push_back(c);
      face_dir.push_back(0);
      kcu[c] = kcuv_of(kcs[c], kcs[OFF(n, m + 1)]);
    }
    if (act(n + 1, m)) {
      face_off.push_back(c);
      face_dir.push_back(1);
      kcv[c] = kcuv_of(kcs[c], kcs[OFF(n + 1, m)]);
    }
  }
  h.npuv = (long long)face_off.size();
  h.face_off = face_off;
  h.face_dir = face_dir;
  // Thin dams: a face whose segment between the two cell centres crosses a
  // dam segment is no momentum face (kcuv = 0, sfincs_quadtree.F90:853-1010).
  // Cells are searched in the dam segment's cell-index box widened by one,
  // as the reference does.  The boundary lists and the advection mask are
  // built from the faces as they were before (the reference applies the dams
  // after initialize_domain); activity and the theta-smoothing neighbour rule
  // see the dams (the reference tests kcuv there at run time).
  RestartData rst;
  std::vector<float> inizs;  // binary ini file (read_zsini_file, sfincs_initial_conditions.F90:270-288)
  if (is_none(K.rstfile) && !is_none(K.inifile)) inizs = read_binary<float>(path(K.inifile), (size_t)h.np);
  if (!is_none(K.rstfile)) {
    rst = read_restart(path(K.rstfile));
    if (rst.type >= 1 && rst.type <= 6) {
      if ((long long)rst.zs.size() != h.np) throw std::runtime_error("restart file: zs has the wrong length");
      if (!rst.q.empty() && (long long)rst.q.size() != h.npuv + 1)
        throw std::runtime_error("restart file: q has the wrong length");
    }
  }
  auto xz = [&](int n, int m) {
    return x0 + cosrot * (1.0f * ((float)m - 0.5f)) * dx - sinrot * (1.0f * ((float)n - 0.5f)) * dy;
  };
  auto yz = [&](int n, int m) {
    return y0 + sinrot * (1.0f * ((float)m - 0.5f)) * dx + cosrot * (1.0f * ((float)n - 0.5f)) * dy;
  };
  // Faces crossed by one polyline: key (dense offset * 2 + 0 for u, 1 for v)
  // -> the last crossing segment (0-based), as the reference records it.
  auto crossed_faces = [&](const std::vector<PolyRow>& pl) {
    std::map<int64_t, int> ind;
    for (size_t ipol = 0; ipol + 1 < pl.size(); ipol++) {
      const float xpa = pl[ipol].x, ypa = pl[ipol].y, xpb = pl[ipol + 1].x, ypb = pl[ipol + 1].y;
      const float xta = cosrot * (xpa - x0) + sinrot * (ypa - y0), yta = -sinrot * (xpa - x0) + cosrot * (ypa - y0);
      const float xtb = cosrot * (xpb - x0) + sinrot * (ypb - y0), ytb = -sinrot * (xpb - x0) + cosrot * (ypb - y0);
      const int na = (int)(yta / dy) + 1, ma = (int)(xta / dx) + 1, nb = (int)(ytb / dy) + 1, mb = (int)(xtb / dx) + 1;
      for (int m = std::max(std::min(ma, mb) - 1, 1); m <= std::min(std::max(ma, mb) + 1, mmax); m++) {
        for (int n = std::max(std::min(na, nb) - 1, 1); n <= std::min(std::max(na, nb) + 1, nmax); n++) {
          if (!act(n, m)) continue;
          const int64_t c = OFF(n, m);
          if (act(n, m + 1) && segments_cross(xpa, ypa, xpb, ypb, xz(n, m), yz(n, m), xz(n, m + 1), yz(n, m + 1)))
            ind[c * 2] = (int)ipol;
          if (act(n + 1, m) && segments_cross(xpa, ypa, xpb, ypb, xz(n, m), yz(n, m), xz(n + 1, m), yz(n + 1, m)))
            ind[c * 2 + 1] = (int)ipol;
        }
      }
    }
    return ind;
  };
  std::vector<uint8_t> dam_u, dam_v;
  if (!is_none(K.thdfile)) {
    dam_u.assign(NA, 0);
    dam_v.assign(NA, 0);
    for (const auto& pl : read_polylines(path(K.thdfile), 0))
      for (const auto& e : crossed_faces(pl)) ((e.first & 1) ? dam_v : dam_u)[e.first >> 1] = 1;
  }
  // cross-sections (sfincs_crosssections.f90:8-127): the crossed uv points in
  // uv-point order, the sign from the last segment crossing each
  if (!is_none(h.out.crsfile)) {
    std::vector<std::string> names;
    const auto pls = read_polylines(path(h.out.crsfile), 0, &names);
    for (size_t k = 0; k < pls.size(); k++) {
      CrossSection cs;
      cs.name = names[k];
      for (const auto& e : crossed_faces(pls[k])) {
        const int64_t c = e.first >> 1;
        const int dir = (int)(e.first & 1);
        const int n = (int)(c % ld) - kGhostPad, m = (int)(c / ld);
        const int n2 = dir == 0 ? n : n + 1, m2 = dir == 0 ? m + 1 : m;
        const auto& a = pls[k][(size_t)e.second];
        const auto& b = pls[k][(size_t)e.second + 1];
        cs.faces.push_back(CrsFace{c, dir, crossing_sign(xz(n, m), yz(n, m), xz(n2, m2), yz(n2, m2), a.x, a.y, b.x, b.y, P.pi),
                                   dir == 0 ? dy : dx});
      }
      h.out.crs.push_back(std::move(cs));
    }
  }

  // ---- bathymetry (regular) or subgrid tables -----------------------------------
  std::vector<float> sg_level_raw;  // z_level as read, [np][levels]
  h.zb_cmp.assign(h.np, 0.0f);
  h.zmin_cmp.assign(h.np, 0.0f);
  if (!P.subgrid) {
    auto zbc = read_binary<float>(path(depfile), (size_t)h.np);
    h.zb.assign(NA, 0.0f);
    for (long long i = 0; i < h.np; i++) {
      h.zb[h.cmp_off[i]] = zbc[i];
      h.zb_cmp[i] = zbc[i];
    }
    h.zbmx_u.assign(NA, 0.0f);
    h.zbmx_v.assign(NA, 0.0f);
    for (size_t f = 0; f < face_off.size(); f++) {
      const int64_t c = face_off[f];
      const int64_t cu = face_dir[f] == 0 ? c + ld : c + 1;
      (face_dir[f] == 0 ? h.zbmx_u : h.zbmx_v)[c] = std::max(h.zb[c], h.zb[cu]) + P.huthresh;
    }
  } else {
    NcFile nc(path(sbgfile));
    const int L = (int)nc.dim("levels");
    if (L < 2) throw std::runtime_error("subgrid tables need at least two levels");
    if (L > kMaxSubgridLevels) throw std::runtime_error("subgrid tables with more than 254 levels are not supported");
    P.nlev = L;
    auto zmin = nc.floats("z_zmin"), zmax = nc.floats("z_zmax"), volmax = nc.floats("z_volmax"),
         zlev = nc.floats("z_level"), uzmin = nc.floats("uv_zmin"), uzmax = nc.floats("uv_zmax"),
         uffit = nc.floats("uv_ffit"), unavg = nc.floats("uv_navg"), uhavg = nc.floats("uv_havg"),
         unrep = nc.floats("uv_nrep"), upwet = nc.floats("uv_pwet");
    if ((long long)zmin.size() != h.np || (long long)uzmin.size() != h.npuv)
      throw std::runtime_error("subgrid file dimensions do not match the mesh (np/npuv)");
    sg_level_raw = zlev;
    // sfincs_subgrid.F90:276-446: read, convert n -> g n^2, and condition the tables
    for (long long f = 0; f < h.npuv; f++) uzmax[f] = std::max(uzmax[f], uzmin[f] + 0.01f);
    for (long long f = 0; f < h.npuv; f++) {
      const int64_t c = face_off[f];
      const int64_t cu = face_dir[f] == 0 ? c + ld : c + 1;
      const float zn = zmin[cmp_of[c]], znu = zmin[cmp_of[cu]];
      if (zn > uzmin[f]) {
        uzmin[f] = std::max(uzmin[f], zn);
        uzmax[f] = std::max(uzmax[f], uzmin[f] + 0.01f);
      }
      if (znu > uzmin[f]) {
        uzmin[f] = std::max(uzmin[f], znu);
        uzmax[f] = std::max(uzmax[f], uzmin[f] + 0.01f);
      }
    }
    for (long long i = 0; i < h.np; i++)
      if (zmax[i] - zmin[i] <= 0.0f) zmax[i] = zmax[i] + 0.01f;
    for (long long f = 0; f < h.npuv; f++)
      if (uzmax[f] - uzmin[f] < 1.0e-7f) uzmax[f] = uzmax[f] + 0.01f;
    h.zz_min.assign(NA, 0.0f);
    h.zz_max.assign(NA, 0.0f);
    h.zz_volmax.assign(NA, 0.0f);
    h.zlev.assign((size_t)(L - 1) * NA, make_float2(0.0f, 0.0f));
    for (long long i = 0; i < h.np; i++) {
      const int64_t c = h.cmp_off[i];
      h.zz_min[c] = zmin[i];
      h.zz_max[c] = zmax[i];
      h.zz_volmax[c] = volmax[i];
      h.zmin_cmp[i] = zmin[i];
      for (int k = 0; k < L - 1; k++) {
        const float a = zlev[(size_t)i * L + k], b = zlev[(size_t)i * L + k + 1];
        h.zlev[(size_t)k * NA + c] = make_float2(a, b - a);
      }
    }
    h.sgz_u.assign(NA, make_float2(0, 0));
    h.sgz_v.assign(NA, make_float2(0, 0));
    h.sgw_u.assign(NA, make_float4(0, 0, 0, 0));
    h.sgw_v.assign(NA, make_float4(0, 0, 0, 0));
    h.rec_u.assign((size_t)(L - 1) * NA, UvRec{});
    h.rec_v.assign((size_t)(L - 1) * NA, UvRec{});
    std::vector<float> hv(L), nv(L), pv(L);
    for (long long f = 0; f < h.npuv; f++) {
      const int64_t c = face_off[f];
      const bool isu = face_dir[f] == 0;
      for (int k = 0; k < L; k++) {
        hv[k] = uhavg[(size_t)f * L + k];
        const float nr = std::max(unrep[(size_t)f * L + k], 0.0001f);
        nv[k] = P.g * (nr * nr);
        pv[k] = upwet[(size_t)f * L + k];
      }
      const float na = std::max(unavg[f], 0.0001f);
      const float navg_w = P.g * (na * na);
      (isu ? h.sgz_u : h.sgz_v)[c] = make_float2(uzmin[f], uzmax[f]);
      (isu ? h.sgw_u : h.sgw_v)[c] = make_float4(hv[L - 1] - uzmax[f], nv[L - 1], navg_w, uffit[f]);
      auto& rec = isu ? h.rec_u : h.rec_v;
      for (int k = 0; k < L - 1; k++) {
        UvRec r{};
        r.havg = hv[k];
        r.dhavg = hv[k + 1] - hv[k];
        r.nrep = nv[k];
        r.dnrep = nv[k + 1] - nv[k];
        r.pwet = pv[k];
        r.dpwet = pv[k + 1] - pv[k];
        rec[(size_t)k * NA + c] = r;
      }
    }
  }

  // ---- boundaries (sfincs_domain.f90:1765-1958) -----------------------------------
  std::vector<int32_t> gb_index(NA, -1);
  std::vector<int32_t> gb_cell;
  bool water_level_bnd = false;
  for (long long i = 0; i < h.np; i++) {
    const int64_t c = h.cmp_off[i];
    const int k = kcs[c];
    if (k == 2 || k == 3 || k == 5 || k == 6) {
      gb_index[c] = (int32_t)gb_cell.size();
      gb_cell.push_back((int32_t)c);
      h.gb_cmp.push_back((int32_t)i);
      if (k == 2) water_level_bnd = true;
    }
  }
  const size_t ngb = gb_cell.size();
  std::vector<int> gb_i1(ngb, 0), gb_i2(ngb, 0), gb_nmi(ngb, -1);
  std::vector<float> gb_fac(ngb, 0.0f), gb_zfix(ngb, 0.0f);
  // kcuv==2/6 faces in reference ip order; outflow (kcs==3) levels are fixed here
  struct KB {
    int64_t face, nmb, nmi;
    int8_t dir, sign;
  };
  std::vector<KB> kb_all;
  for (size_t f = 0; f < face_off.size(); f++) {
    const int64_t c = face_off[f];
    const int8_t kc = face_dir[f] == 0 ? kcu[c] : kcv[c];
    if (kc != 2 && kc != 6) continue;
    const int64_t cu = face_dir[f] == 0 ? c + ld : c + 1;
    KB e;
    e.face = c;
    e.dir = face_dir[f];
    if (kcs[c] == 1) {
      e.nmb = cu;
      e.nmi = c;
      e.sign = -1;
    } else {
      e.nmb = c;
      e.nmi = cu;
      e.sign = 1;
    }
    if (kcs[e.nmb] == 3) gb_zfix[gb_index[e.nmb]] = P.subgrid ? h.zz_min[e.nmb] : h.zb[e.nmb];
    kb_all.push_back(e);
  }

  // ---- boundary conditions files (sfincs_boundaries.f90:8-213) ----------------------
  int nbnd = 0;
  std::vector<float> xb, yb;
  read_boundary_series(h, K, water_level_bnd, xb, yb, nbnd);

  // ---- downstream river points (sfincs_boundaries.f90:217-270): the cell of each
  // point's internal point and the level drop slope * distance to it
  bool river = false;
  for (size_t ib = 0; ib < ngb; ib++) river = river || kcs[gb_cell[ib]] == 5;
  std::vector<float> xr, yr, dzr;
  std::vector<int32_t> zsir;
  if (river) {
    if (is_none(K.bdrfile)) throw std::runtime_error("downstream river points (msk 5) need a bdrfile");
    for (const auto& r : read_table(path(K.bdrfile))) {
      if (r.size() < 6) throw std::runtime_error("bdrfile: expected x y x_internal y_internal slope distance");
      const float x = (float)r[0], y = (float)r[1], xin = (float)r[2], yin = (float)r[3];
      const float slope = (float)r[4], dist = (float)r[5];
      // the cell holding the internal point (find_quadtree_cell on the regular grid)
      const float xt = cosrot * (xin - x0) + sinrot * (yin - y0), yt = -sinrot * (xin - x0) + cosrot * (yin - y0);
      const int n = (int)(yt / dy) + 1, m = (int)(xt / dx) + 1;
      if (!act(n, m)) throw std::runtime_error("bdrfile: internal point outside the active grid");
      xr.push_back(x);
      yr.push_back(y);
      zsir.push_back((int32_t)OFF(n, m));
      dzr.push_back(dist < 0.0f ? -slope * std::sqrt((xin - x) * (xin - x) + (yin - y) * (yin - y)) : -slope * dist);
    }
    if (xr.empty()) throw std::runtime_error("bdrfile holds no points");
  }
  std::vector<int> gb_bdr(ngb, -1);

  // ---- find_boundary_indices (sfincs_boundaries.f90:455-679) -------------------------
  if (ngb > 0 && (nbnd > 0 || river)) {
    for (size_t ib = 0; ib < ngb; ib++) {
      const int64_t c = gb_cell[ib];
      const long long ic = cmp_of[c];
      const float x = h.z_xz[ic], y = h.z_yz[ic];
      if (kcs[c] == 2) {
        if (nbnd > 1) {
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
      } else if (kcs[c] == 5) {  // nearest point of the bdr file (:596-613)
        float dst1 = 1.0e10f;
        for (size_t j = 0; j < xr.size(); j++) {
          const float ddx = xr[j] - x, ddy = yr[j] - y;
          const float dst = std::sqrt(ddx * ddx + ddy * ddy);
          if (dst < dst1) {
            dst1 = dst;
            gb_bdr[ib] = (int)j;
          }
        }
      } else if (kcs[c] == 6) {
        const int n = h.z_n[ic], m = h.z_m[ic];
        const int cand[4][2] = {{n, m + 1}, {n + 1, m}, {n, m - 1}, {n - 1, m}};
        int32_t nmi = -1;
        for (auto& q : cand)
          if (act(q[0], q[1]) && kcs[OFF(q[0], q[1])] == 1) nmi = (int32_t)OFF(q[0], q[1]);
        if (nmi < 0)
          kcs[c] = 0;  // isolated Neumann cell reset to inactive (sfincs_boundaries.f90:661-672)
        else
          gb_nmi[ib] = nmi;
      }
    }
  }
  for (size_t ib = 0; ib < ngb; ib++)
    if (kcs[gb_cell[ib]] == 6 && gb_nmi[ib] >= 0) h.neu.push_back(make_int2(gb_cell[ib], gb_nmi[ib]));
  if (!rst.uvmean.empty() && rst.uvmean.size() != kb_all.size())
    throw std::runtime_error("restart file: uvmean has the wrong length");
  h.kb_bface.assign(kb_all.size(), -1);
  for (size_t ib_ref = 0; ib_ref < kb_all.size(); ib_ref++) {
    const auto& e = kb_all[ib_ref];
    if (kcs[e.nmb] == 6) continue;  // lateral Neumann faces are updated by the momentum kernel
    h.kb_bface[ib_ref] = (int)h.bfaces.size();
    if (!rst.uvmean.empty()) {
      h.uvmean0.resize(h.bfaces.size() + 1, 0.0f);
      h.uvmean0.back() = rst.uvmean[ib_ref];
    }
    const int ib = gb_index[e.nmb];
    BndFace b{};
    b.face = (int)e.face;
    b.nmb = (int)e.nmb;
    b.nmi = (int)e.nmi;
    b.info = (e.dir == 1 ? 1 : 0) | (e.sign > 0 ? 2 : 0) | (kcs[e.nmb] == 3 ? 4 : 0) | (nbnd > 1 ? 8 : 0);
    b.i1 = gb_i1[ib];
    b.i2 = gb_i2[ib];
    b.fac = gb_fac[ib];
    b.zbuv = P.subgrid ? 0.0f : 0.5f * (h.zb[e.face] + h.zb[e.dir == 0 ? e.face + ld : e.face + 1]);
    b.floor = P.subgrid ? h.zz_min[e.nmb] : h.zb[e.nmb];
    b.zfix = gb_zfix[ib];
    b.len = P.geo ? (e.dir == 1 ? h.geo_dxm[b.nmi] : P.geo_dyrm) : (e.dir == 1 ? dx : dy);
    if (kcs[e.nmb] == 2 && nbnd == 0) b.info |= 4, b.zfix = 0.0f;  // no boundary data: zsb stays 0
    // an isolated Neumann cell reset to inactive keeps its lateral face in the
    // boundary list, where its level zsb stays at its initial 0 (sfincs_boundaries.f90:661-672, 800-921)
    if (kcs[e.nmb] == 0) b.info |= 4, b.zfix = 0.0f;
    if (kcs[e.nmb] == 5) {  // downstream river cell: level from its internal point
      const int j = gb_bdr[ib];
      if (j < 0) throw std::runtime_error("downstream river cell without a bdr point");
      b.info = (b.info & ~8) | 32;
      b.zsi = zsir[(size_t)j];
      b.zfix = dzr[(size_t)j];
      b.i1 = b.i2 = 0;
    }
    h.bfaces.push_back(b);
  }
  h.dense2cmp = cmp_of;
  h.x0 = x0;
  h.y0 = y0;
  h.cosrot = cosrot;
  h.sinrot = sinrot;
  P.ngbnd = (int)ngb;
  P.nkcuv2 = (int)h.bfaces.size();
  P.nneu = (int)h.neu.size();

  // ---- roughness (sfincs_domain.f90:1960-2061) -------------------------------------------
  if (!P.subgrid) {
    h.gn2_u.assign(NA, 9.81f * 0.02f * 0.02f);
    h.gn2_v.assign(NA, 9.81f * 0.02f * 0.02f);
    std::vector<float> rgh;
    if (!is_none(manningfile)) rgh = read_binary<float>(path(manningfile), (size_t)h.np);
    const float gn2land = manning_land < 0.0f ? 9.81f * (manning * manning) : 9.81f * (manning_land * manning_land);
    const float gn2sea = manning_sea < 0.0f ? 9.81f * (manning * manning) : 9.81f * (manning_sea * manning_sea);
    for (size_t f = 0; f < face_off.size(); f++) {
      const int64_t c = face_off[f];
      const bool isu = face_dir[f] == 0;
      const int64_t cu = isu ? c + ld : c + 1;
      if ((isu ? kcu[c] : kcv[c]) <= 0) continue;
      float val;
      if (!rgh.empty()) {
        const float a = 0.5f * (rgh[cmp_of[c]] + rgh[cmp_of[cu]]);
        val = 9.81f * (a * a);
      } else {
        const float zbuv = 0.5f * (h.zb[c] + h.zb[cu]);
        val = zbuv > rghlevland ? gn2land : gn2sea;
      }
      (isu ? h.gn2_u : h.gn2_v)[c] = val;
    }
  }

  // ---- infiltration con/c2d (sfincs_infiltration.f90:8-606) ---------------------------------
  P.infiltration = 0;
  if (P.precip) {
    if (qinf > 0.0f) {
      P.infiltration = 1;
      h.qinf.assign(NA, 0.0f);
      for (long long i = 0; i < h.np; i++) {
        const int64_t c = h.cmp_off[i];
        const float zz = P.subgrid ? h.zz_min[c] : h.zb[c];
        h.qinf[c] = zz > qinf_zmin ? qinf : 0.0f;
      }
    } else if (!is_none(qinffile)) {
      P.infiltration = 1;
      h.qinf.assign(NA, 0.0f);
      auto r = read_binary<float>(path(qinffile), (size_t)h.np);
      for (long long i = 0; i < h.np; i++) h.qinf[h.cmp_off[i]] = r[i] / 3600.0f / 1000.0f;
    }
  }
  load_infiltration_models(h, K, NA, h.cmp_off);
  apply_restart_infiltration(h, rst, h.cmp_off);

  // ---- weirs (sfincs_structures.f90:38-381) ----------------------------------------
  // Every face a weir polyline crosses gets the crossed length (the face's
  // corner-to-corner segment projected onto the weir segment), the larger
  // crest level and the discharge coefficient interpolated at the face centre
  // between the segment's end points.  Faces whose crest is above the face
  // bed (zbuvmx, or the subgrid uv_zmin) become weir faces (kcuv = 3).  The
  // face centre and corners use half the face width along both axes, as the
  // reference does (exact for dx = dy).
  std::vector<uint8_t> weir_u, weir_v;
  if (!is_none(K.weirfile)) {
    weir_u.assign(NA, 0);
    weir_v.assign(NA, 0);
    struct Acc {
      float len = 0.0f, height = -9999.0f, cd = 0.0f;
    };
    std::map<int64_t, Acc> acc;
    const float pi = P.pi;
    for (const auto& pl : read_polylines(path(K.weirfile), 2)) {
      for (const auto& e : crossed_faces(pl)) {
        const int64_t c = e.first >> 1;
        const int dir = (int)(e.first & 1), ipol = e.second;
        const int m = (int)(c / ld), n = (int)(c % ld) - kGhostPad;
        const float dxs = dir == 0 ? dy : dx;
        float xuv, yuv, xuv1, yuv1, xuv2, yuv2;
        if (dir == 0) {
          xuv = xz(n, m) + 0.5f * dxs * std::cos(rotation);
          yuv = yz(n, m) + 0.5f * dxs * std::sin(rotation);
          xuv1 = xuv + 0.5f * dxs * std::cos(rotation - 0.5f * pi);
          yuv1 = yuv + 0.5f * dxs * std::sin(rotation - 0.5f * pi);
          xuv2 = xuv + 0.5f * dxs * std::cos(rotation + 0.5f * pi);
          yuv2 = yuv + 0.5f * dxs * std::sin(rotation + 0.5f * pi);
        } else {
          xuv = xz(n, m) + 0.5f * dxs * std::cos(rotation + 0.5f * pi);
          yuv = yz(n, m) + 0.5f * dxs * std::sin(rotation + 0.5f * pi);
          xuv1 = xuv + 0.5f * dxs * std::cos(rotation - pi);
          yuv1 = yuv + 0.5f * dxs * std::sin(rotation - pi);
          xuv2 = xuv + 0.5f * dxs * std::cos(rotation);
          yuv2 = yuv + 0.5f * dxs * std::sin(rotation);
        }
        const PolyRow &r0 = pl[(size_t)ipol], &r1 = pl[(size_t)ipol + 1];
        Acc& a = acc[e.first];
        a.len = a.len + projected_length(xuv1, yuv1, xuv2, yuv2, r0.x, r0.y, r1.x, r1.y);
        const float dst1 = std::sqrt((xuv - r0.x) * (xuv - r0.x) + (yuv - r0.y) * (yuv - r0.y));
        const float dst2 = std::sqrt((xuv - r1.x) * (xuv - r1.x) + (yuv - r1.y) * (yuv - r1.y));
        const float wfac = dst1 / (dst1 + dst2);
        a.height = std::max(a.height, r0.p[0] * (1.0f - wfac) + r1.p[0] * wfac);
        a.cd = r0.p[1] * (1.0f - wfac) + r1.p[1] * wfac;
      }
    }
    for (const auto& e : acc) {
      const int64_t c = e.first >> 1;
      const int dir = (int)(e.first & 1);
      const float bed = P.subgrid ? (dir == 0 ? h.sgz_u : h.sgz_v)[c].x : (dir == 0 ? h.zbmx_u : h.zbmx_v)[c];
      if (!(e.second.height > bed)) continue;
      StrucFace w{};
      w.face = (int)c;
      w.nm = (int)c;
      w.nmu = (int)(dir == 0 ? c + ld : c + 1);
      w.dir = dir;
      w.height = e.second.height;
      w.cd = e.second.cd;
      w.len = e.second.len / (dir == 0 ? dy : dx);
      h.struc.push_back(w);
      (dir == 0 ? weir_u : weir_v)[c] = 1;
    }
    // a weir on a water-level boundary face: no boundary flux there (sfincs_boundaries.f90:1009)
    for (auto& b : h.bfaces)
      if ((b.info & 1 ? weir_v : weir_u)[b.face]) b.info |= 16;
  }
  P.nstruc = (int)h.struc.size();

  // ---- flags, advection mask, theta smoothing -----------------------------------------------
  h.flags.assign(NA, 0);
  auto KU = [&](int n, int m) -> int { return (n >= 1 && n <= nmax && m >= 1 && m <= mmax) ? kcu[OFF(n, m)] : 0; };
  auto KV = [&](int n, int m) -> int { return (n >= 1 && n <= nmax && m >= 1 && m <= mmax) ? kcv[OFF(n, m)] : 0; };
  // kcuv after the thin dams (0) and the weirs (3, applied after the dams)
  auto after_structures = [&](int n, int m, int k, const std::vector<uint8_t>& weir, const std::vector<uint8_t>& dam) {
    if (n < 1 || n > nmax || m < 1 || m > mmax) return k;
    if (!weir.empty() && weir[OFF(n, m)]) return 3;
    if (!dam.empty() && dam[OFF(n, m)]) return 0;
    return k;
  };
  auto KUd = [&](int n, int m) -> int { return after_structures(n, m, KU(n, m), weir_u, dam_u); };
  auto KVd = [&](int n, int m) -> int { return after_structures(n, m, KV(n, m), weir_v, dam_v); };
  const bool do_mask = P.advection && advection_mask && nmax > 1;
  for (long long i = 0; i < h.np; i++) {
    const int n = h.z_n[i], m = h.z_m[i];
    const int64_t c = OFF(n, m);
    uint16_t f = F_ACT;
    if (kcs[c] == 1) f |= F_KCS1;
    const int ku = kcu[c], kv = kcv[c];
    if (KUd(n, m) == 1 || KUd(n, m) == 6) f |= F_UACT;
    if (KVd(n, m) == 1 || KVd(n, m) == 6) f |= F_VACT;
    const bool cdn = act(n - 1, m), cup = act(n + 1, m), clf = act(n, m - 1), crt = act(n, m + 1);
    if (cdn) f |= F_CDN;
    if (cup) f |= F_CUP;
    if (clf) f |= F_CLF;
    if (crt) f |= F_CRT;
    if (P.advection) {  // sfincs_domain.f90:2147-2178
      bool madv_u = true, madv_v = true;
      if (do_mask) {
        const int u_ndm = cdn ? KU(n - 1, m) : ku, u_num = cup ? KU(n + 1, m) : ku;
        madv_u = KU(n, m + 1) == 1 && KU(n, m - 1) == 1 && KV(n, m) == 1 && KV(n, m + 1) == 1 && KV(n - 1, m) == 1 &&
                 KV(n - 1, m + 1) == 1 && u_ndm == 1 && u_num == 1;
        const int v_ndm = clf ? KV(n, m - 1) : kv, v_num = crt ? KV(n, m + 1) : kv;
        madv_v = KV(n + 1, m) == 1 && KV(n - 1, m) == 1 && KU(n, m) == 1 && KU(n + 1, m) == 1 && KU(n, m - 1) == 1 &&
                 KU(n + 1, m - 1) == 1 && v_ndm == 1 && v_num == 1;
      }
      if (madv_u) f |= F_UADV;
      if (madv_v) f |= F_VADV;
    }
    if (KUd(n, m - 1) == 1 && KUd(n, m + 1) == 1) f |= F_UTH;  // kcuv(u_nmd)==1 and kcuv(u_nmu)==1
    if (KVd(n - 1, m) == 1 && KVd(n + 1, m) == 1) f |= F_VTH;
    h.flags[c] = f;
  }
  h.kcs_cmp.resize(h.np);
  for (long long i = 0; i < h.np; i++) {
    h.kcs_cmp[i] = kcs[h.cmp_off[i]];
    if (kcs[h.cmp_off[i]] == 1) {
      h.n_kcs1++;
      h.area_total_kcs1 += (double)(P.geo ? h.geo_area[h.cmp_off[i]] : P.area);
    }
  }

  // ---- initial conditions (sfincs_initial_conditions.F90:98-106, sfincs_subgrid.F90:907-962) --
  h.zs.assign(NA, 0.0f);
  for (long long i = 0; i < h.np; i++) {
    const int64_t c = h.cmp_off[i];
    const float base = P.subgrid ? h.zz_min[c] : h.zb[c];
    // inizs (real*8) from the real*4 restart or ini file, else zini
    const double ini = !rst.zs.empty() ? (double)rst.zs[i] : (!inizs.empty() ? (double)inizs[i] : (double)P.zini);
    h.zs[c] = (float)std::max((double)base, ini);
  }
  h.zsmax.assign(NA, -999.0f);
  // initial fluxes from a restart file, and the velocities they imply
  // (sfincs_initial_conditions.F90:110-173), in both ping-pong buffers
  if (!rst.q.empty()) {
    h.q0u.assign(NA, 0.0f);
    h.q0v.assign(NA, 0.0f);
    h.uv0u.assign(NA, 0.0f);
    h.uv0v.assign(NA, 0.0f);
    h.kf0u.assign(NA, 0);
    h.kf0v.assign(NA, 0);
    for (size_t f = 0; f < face_off.size(); f++) {
      const int64_t c = face_off[f];
      const int dir = face_dir[f];
      const int64_t cu = dir == 0 ? c + ld : c + 1;
      const float q = rst.q[f];
      (dir == 0 ? h.q0u : h.q0v)[c] = q;
      if (q != 0.0f) (dir == 0 ? h.kf0u : h.kf0v)[c] = KF_STALE | KF_WET2;
      const float zsuv = std::max(h.zs[c], h.zs[cu]);
      float huv = 0.0f;
      if (P.subgrid) {
        const float2 zr = (dir == 0 ? h.sgz_u : h.sgz_v)[c];
        if (!(zsuv > zr.x + P.huthresh)) continue;
        if (zsuv > zr.y - 1.0e-4f) {
          huv = (dir == 0 ? h.sgw_u : h.sgw_v)[c].x + zsuv;
        } else {
          const float dzuv = (zr.y - zr.x) / (float)(P.nlev - 1);
          const int iuv = (int)((zsuv - zr.x) / dzuv) + 1;
          const float facint = (zsuv - (zr.x + (float)(iuv - 1) * dzuv)) / dzuv;
          const UvRec& r = (dir == 0 ? h.rec_u : h.rec_v)[(size_t)(iuv - 1) * NA + (size_t)c];
          huv = r.havg + r.dhavg * facint;
        }
        huv = std::max(huv, P.huthresh);
      } else {
        if (!(zsuv > (dir == 0 ? h.zbmx_u : h.zbmx_v)[c])) continue;
        huv = std::max(zsuv - 0.5f * (h.zb[c] + h.zb[cu]), P.huthresh);
      }
      (dir == 0 ? h.uv0u : h.uv0v)[c] = std::max(std::min(q / huv, 4.0f), -4.0f);
    }
  }
  if (P.wiggle) h.zs0 = h.zs;
  if (P.subgrid) {
    const int L = P.nlev;
    h.zvol.assign(NA, 0.0);
    h.vneg.assign(NA, 0);
    for (long long i = 0; i < h.np; i++) {
      const int64_t c = h.cmp_off[i];
      const double zs = h.zs[c];
      if (zs >= (double)h.zz_max[c]) {
        h.zvol[c] = (double)h.zz_volmax[c] + (double)(P.geo ? h.geo_area[c] : P.area) *
                                                 (zs - (double)std::max(h.zz_max[c], -20.0f));
      } else {
        const float* dep = &sg_level_raw[(size_t)i * L];  // z_level of this cell, levels 1..L
        int ivol = 1;
        for (int il = 2; il <= L; il++) {
          if ((double)dep[il - 1] > zs) {
            ivol = il - 1;
            break;
          }
        }
        const float dzvol = h.zz_volmax[c] / (float)(L - 1);
        const float facint =
            (float)((zs - (double)dep[ivol - 1]) / (double)std::max(dep[ivol] - dep[ivol - 1], 0.001f));
        h.zvol[c] = (double)((float)(ivol - 1) * dzvol + facint * dzvol);
      }
      h.vneg[c] = h.zvol[c] < 0.0 ? 1 : 0;
    }
  }

  // ---- meteo time series and Cd table (sfincs_meteo.f90:247-327) ------------------------------
  read_meteo_series(h, K, rotation);

  // ---- point sources (sfincs_discharges.f90:8-324) ------------------------------------------------
  if (!is_none(srcfile)) {
    auto xy = read_table(path(srcfile));
    auto tb = read_table(path(disfile));
    const int nsrc = (int)xy.size();
    for (auto& r : xy) {
      const float x = (float)r.at(0), y = (float)r.at(1);
      const float xt = cosrot * (x - x0) + sinrot * (y - y0);
      const float yt = -sinrot * (x - x0) + cosrot * (y - y0);
      const int n = (int)(yt / dy) + 1, m = (int)(xt / dx) + 1;  // sfincs_quadtree.F90:788-790
      if (!act(n, m)) throw std::runtime_error("point source outside the active mesh");
      h.src_cell.push_back((int32_t)OFF(n, m));
    }
    for (auto& r : tb) {
      if ((int)r.size() < nsrc + 1) throw std::runtime_error("dis file has fewer columns than src points");
      h.tsrc.push_back((float)r[0]);
      for (int is = 0; is < nsrc; is++) h.qsrc.push_back((float)r[is + 1]);
    }
    P.nsrc = nsrc;
    P.ntsrc = (int)h.tsrc.size();
  }
  // drainage structures (sfincs_discharges.f90:70-320): one line each,
  // "x_intake y_intake x_outfall y_outfall type params...", the intake and
  // outfall cells appended after the point sources
  if (!is_none(K.drnfile)) {
    auto cell_of = [&](float x, float y) -> int64_t {
      const float xt = cosrot * (x - x0) + sinrot * (y - y0);
      const float yt = -sinrot * (x - x0) + cosrot * (y - y0);
      const int n = (int)(yt / dy) + 1, m = (int)(xt / dx) + 1;  // sfincs_quadtree.F90:788-790
      if (!act(n, m)) throw std::runtime_error("drainage point outside the active mesh");
      return OFF(n, m);
    };
    for (const DrnLine& r : read_drainage(path(K.drnfile))) {
      DrnDev d{};
      d.type = r.type;
      const int64_t ci = cell_of(r.xs, r.ys), co = cell_of(r.xo, r.yo);
      d.cin = (int)ci;
      d.cout = (int)co;
      for (int k = 0; k < 6; k++) d.p[k] = r.p[k];
      const int ni = (int)(ci % ld) - kGhostPad, mi = (int)(ci / ld), no = (int)(co % ld) - kGhostPad, mo = (int)(co / ld);
      const float xsnk = xz(ni, mi), ysnk = yz(ni, mi), xsrc = xz(no, mo), ysrc = yz(no, mo);
      d.distance = std::sqrt((xsrc - xsnk) * (xsrc - xsnk) + (ysrc - ysnk) * (ysrc - ysnk));
      h.drn.push_back(d);
      h.src_cell.push_back((int32_t)ci);
      h.src_cell.push_back((int32_t)co);
    }
  }
  P.ndrn = (int)h.drn.size();
  // 32 x 8 cell tiles that hold at least one active cell (the work list of the
  // cell kernels; a runner concatenates the lists of its models)
  for (int m0 = 1; m0 <= P.mmax; m0 += 8)
    for (int n0 = 1; n0 <= P.nmax; n0 += 32) {
      bool any = false;
      for (int m = m0; m < m0 + 8 && m <= P.mmax && !any; m++)
        for (int n = n0; n < n0 + 32 && n <= P.nmax; n++)
          if (h.flags[(size_t)m * P.ld + kGhostPad + n] & F_ACT) {
            any = true;
            break;
          }
      if (any) h.tiles.push_back(int2{n0, m0});
    }
  read_obs_points(h);
  return H;
}

// ============================================================================
// DeviceModel
// ============================================================================
// Device residency in ONE allocation: the layout pass below runs twice, first
// to size every array (256-byte aligned sub-allocations), then to place and
// upload them.  device_bytes_needed() runs only the first pass, so admission
// control knows a model's footprint before anything is allocated.
namespace {
struct Placer {
  char* base = nullptr;  // null: sizing pass
  size_t off = 0;
  template <class X>
  X* take(size_t n) {
    if (n == 0) return nullptr;
    off = (off + 255) & ~(size_t)255;
    X* p = base ? reinterpret_cast<X*>(base + off) : nullptr;
    off += n * sizeof(X);
    return p;
  }
};
}  // namespace

template <class F>
static void place_model(const HostModel& h, ScnDev& d, int32_t*& cmp, int32_t*& qmu, int32_t*& qmv, Placer& pl,
                        F&& fill) {
  const size_t NA = (size_t)h.p.nalloc;
  auto up = [&](auto& dst, const auto& v) {
    using X = typename std::decay_t<decltype(v)>::value_type;
    X* q = pl.template take<X>(v.size());
    if (q) fill(q, v.data(), v.size() * sizeof(X));
    dst = q;
  };
  auto zero = [&](auto& dst, size_t n) {
    using X = std::remove_const_t<std::remove_pointer_t<std::decay_t<decltype(dst)>>>;
    X* q = pl.template take<X>(n);
    if (q) fill(q, nullptr, n * sizeof(X));
    dst = q;
  };
  // store variables (sfincs_domain.f90:2296-2310): vmax and t_zsmax start at
  // -999, twet at 0; qmax at 0 (the reference allocates it without a value)
  auto place_store = [&](size_t n) {
    auto filled = [&](float*& dst, bool on, float v) {
      if (on) up(dst, std::vector<float>(n, v));
      else dst = nullptr;
    };
    filled(d.vmax, h.p.store_vmax, -999.0f);
    filled(d.qmax, h.p.store_qmax, 0.0f);
    filled(d.twet, h.p.store_twet, 0.0f);
    filled(d.tzsmax, h.p.store_tzsmax, -999.0f);
  };
  if (h.p.quadtree) {
    // compact cells (npc), uv points (npuv) and q/uv arrays (npuv + ncuv + dummy)
    const size_t NC = (size_t)h.np, NF = (size_t)h.npuv, NQ = (size_t)(h.npuv + h.p.ncuv + 1);
    up(d.zs, h.zs);
    up(d.zsmax, h.zsmax);
    place_store(NC);
    up(d.zvol, h.zvol);
    if (h.p.wiggle) {
      up(d.zs0, h.zs0);
      zero(d.zsderv, NC);
    } else {
      d.zs0 = nullptr;
      d.zsderv = nullptr;
    }
    zero(d.kf[0], NF);
    d.kf[1] = d.kf[0];
    if (h.p.subgrid) up(d.vneg, h.vneg);
    else d.vneg = nullptr;
    for (int b = 0; b < 2; b++) {
      if (h.q0u.empty()) {
        zero(d.qu[b], NQ);
        zero(d.uu[b], NQ);
      } else {  // fluxes from a restart file in both buffers
        up(d.qu[b], h.q0u);
        up(d.uu[b], h.uv0u);
      }
      d.qv[b] = d.qu[b];
      d.vv[b] = d.uu[b];
    }
    up(d.flags, h.flags);
    up(d.zb, h.zb);
    d.zbmx_u = d.zbmx_v = d.gn2_u = d.gn2_v = nullptr;
    up(d.zbmx, h.zbmx_q);
    up(d.gn2, h.gn2_q);
    up(d.sgz_u, h.sgz_u);
    d.sgz_v = d.sgz_u;
    up(d.sgw_u, h.sgw_u);
    d.sgw_v = d.sgw_u;
    up(d.rec_u, h.rec_u);
    d.rec_v = d.rec_u;
    up(d.zz_min, h.zz_min);
    up(d.zz_max, h.zz_max);
    up(d.zz_volmax, h.zz_volmax);
    up(d.zlev, h.zlev);
    if (h.p.use_qext) zero(d.qext, NC);
    else d.qext = nullptr;
    up(d.qinf, h.qinf);
    up(d.qface, h.qface);
    up(d.qcell, h.qcell);
    up(d.qcuv, h.qcuv);
    up(d.qlev, h.qlev);
    up(qmu, h.qmap_u);
    up(qmv, h.qmap_v);
    d.rc4_u = d.rc4_v = nullptr;
    d.rc2_u = d.rc2_v = nullptr;
    d.rl_u = d.rl_v = nullptr;
    d.zc = nullptr;
    d.zl = nullptr;
  } else {
    d.qface = nullptr;
    d.qcell = nullptr;
    d.qcuv = nullptr;
    d.qlev = nullptr;
    d.zbmx = d.gn2 = nullptr;
    qmu = qmv = nullptr;
    d.rc4_u = d.rc4_v = nullptr;
    d.rc2_u = d.rc2_v = nullptr;  // set below for subgrid models
    d.rl_u = d.rl_v = nullptr;
    d.zc = nullptr;
    d.zl = nullptr;
  up(d.zs, h.zs);
  up(d.zsmax, h.zsmax);
  place_store(NA);
  up(d.zvol, h.zvol);
  if (h.p.wiggle) {
    up(d.zs0, h.zs0);
    zero(d.zsderv, NA);
  } else {
    d.zs0 = nullptr;
    d.zsderv = nullptr;
  }
  if (h.kf0u.empty()) {
    zero(d.kf[0], NA);
    zero(d.kf[1], NA);
  } else {  // restart fluxes in both buffers: the first dry steps must clear them
    up(d.kf[0], h.kf0u);
    up(d.kf[1], h.kf0v);
  }
  if (h.p.subgrid) up(d.vneg, h.vneg);
  else d.vneg = nullptr;
  for (int b = 0; b < 2; b++) {
    if (h.q0u.empty()) {
      zero(d.qu[b], NA);
      zero(d.qv[b], NA);
      zero(d.uu[b], NA);
      zero(d.vv[b], NA);
    } else {  // a restart file's fluxes
      up(d.qu[b], h.q0u);
      up(d.qv[b], h.q0v);
      up(d.uu[b], h.uv0u);
      up(d.vv[b], h.uv0v);
    }
  }
  up(d.flags, h.flags);
  up(d.zb, h.zb);
  up(d.zbmx_u, h.zbmx_u);
  up(d.zbmx_v, h.zbmx_v);
  up(d.gn2_u, h.gn2_u);
  up(d.gn2_v, h.gn2_v);
  up(d.sgz_u, h.sgz_u);
  up(d.sgz_v, h.sgz_v);
  up(d.sgw_u, h.sgw_u);
  up(d.sgw_v, h.sgw_v);
  up(d.rec_u, h.rec_u);
  up(d.rec_v, h.rec_v);
  up(d.zz_min, h.zz_min);
  up(d.zz_max, h.zz_max);
  up(d.zz_volmax, h.zz_volmax);
  up(d.zlev, h.zlev);
  if (h.p.subgrid) {  // record cache, empty (all codes 0)
    zero(d.rc4_u, NA);
    zero(d.rc4_v, NA);
    zero(d.rc2_u, NA);
    zero(d.rc2_v, NA);
    zero(d.rl_u, NA);
    zero(d.rl_v, NA);
    zero(d.zc, NA);
    zero(d.zl, NA);
  } else {
    d.rc4_u = d.rc4_v = nullptr;
    d.rc2_u = d.rc2_v = nullptr;
    d.rl_u = d.rl_v = nullptr;
    d.zc = nullptr;
    d.zl = nullptr;
  }
  if (h.p.use_qext) zero(d.qext, NA);
  else d.qext = nullptr;
  up(d.qinf, h.qinf);
  }
  up(d.t_bnd, h.t_bnd);
  up(d.zs_bnd, h.zs_bnd);
  up(d.tide_w, h.tide.omega);
  up(d.tide_amp, h.tide.amp);
  up(d.tide_pha, h.tide.phase);
  zero(d.zst_bnd, (size_t)std::max(h.p.nbnd, 1));
  up(d.bfaces, h.bfaces);
  if (h.uvmean0.empty())
    zero(d.uvmean, (size_t)std::max(h.p.nkcuv2, 1));
  else
    up(d.uvmean, h.uvmean0);
  up(d.neu, h.neu);
  up(d.tprcp, h.tprcp);
  up(d.vprcp, h.vprcp);
  up(d.twnd, h.twnd);
  up(d.wmag, h.wmag);
  up(d.wdir, h.wdir);
  up(d.cdval, h.cdval);
  up(d.x73, h.x73);
  {  // gridded meteo: the raw grids, the cell centres, the window fields
    const size_t ncell = h.p.quadtree ? (size_t)h.np : NA;
    for (int kq = 0; kq < 3; kq++) {
      const MeteoGridHost& g = h.mgh[kq];
      MeteoGrid& m = d.mg[kq];
      m = MeteoGrid{};
      m.nt = g.nt;
      m.nrows = g.nrows;
      m.ncols = g.ncols;
      m.x_ll = g.x_ll;
      m.y_ll = g.y_ll;
      m.dx = g.dx;
      m.dy = g.dy;
      up(m.times, g.times);
      up(m.v0, g.v[0]);
      up(m.v1, g.v[1]);
    }
    {  // the spiderweb's records (scalars came with h.p)
      const SpwHost& w = h.spw;
      up(d.spw.times, w.times);
      up(d.spw.xe, w.xe);
      up(d.spw.ye, w.ye);
      up(d.spw.wu, w.wu);
      up(d.spw.wv, w.wv);
      up(d.spw.pabs, h.spw_pabs);
      up(d.spw.prcp, w.precip ? w.prcp : std::vector<float>());
    }
    d.nmeteo = (int)h.np;
    if (h.p.meteo3d) {
      up(d.xz, h.z_xz);
      up(d.yz, h.z_yz);
    } else {
      d.xz = d.yz = nullptr;
    }
    auto field = [&](float*& dst, bool on, float v) {
      if (on) up(dst, std::vector<float>(ncell, v));
      else dst = nullptr;
    };
    const bool wf = h.p.wind_field, pf = h.p.patmos, rf = h.p.prcp_field;
    field(d.tauwu0, wf, 0.0f);
    field(d.tauwu1, wf, 0.0f);
    field(d.tauwv0, wf, 0.0f);
    field(d.tauwv1, wf, 0.0f);
    field(d.patm0, pf, 0.0f);
    field(d.patm1, pf, 0.0f);
    field(d.prcp0, rf, 0.0f);
    field(d.prcp1, rf, 0.0f);
  }
  for (int j = 0; j < 5; j++) {
    up(d.inf_par[j], h.inf_par[j]);
    up(d.inf_st[j], h.inf_st[j]);
  }
  up(d.inf_rain, h.inf_rain);
  up(d.cumprcp, h.cumprcp);
  up(d.geo_dxm, h.geo_dxm);
  up(d.geo_dxminv, h.geo_dxminv);
  up(d.geo_area, h.geo_area);
  up(d.geo_fcor, h.geo_fcor);
  if (h.need_qinfmap)
    zero(d.qinfmap, h.p.quadtree ? (size_t)h.np : NA);
  else
    d.qinfmap = nullptr;
  up(d.cuminf, h.cuminf);
  up(d.tsrc, h.tsrc);
  up(d.qsrc, h.qsrc);
  zero(d.qtsrc, (size_t)std::max(h.p.nsrc + 2 * h.p.ndrn, 1));
  up(d.src_cell, h.src_cell);
  up(d.struc, h.struc);
  up(d.drn, h.drn);
  up(d.drn_status, std::vector<int>(h.drn.size(), 1));          // open
  up(d.drn_frac, std::vector<float>(h.drn.size(), 1.0f));      // fully open
  up(cmp, h.cmp_off);
  d.cmp = h.p.quadtree ? nullptr : cmp;  // compact cell -> storage offset for the meteo fields
  zero(d.st, 1);
}

int cell_index(const HostModel& h, double xd, double yd) {
  if (h.p.quadtree) return quadtree_cell_index(h, xd, yd);
  const float x = (float)xd, y = (float)yd;
  const float xt = h.cosrot * (x - h.x0) + h.sinrot * (y - h.y0);
  const float yt = -h.sinrot * (x - h.x0) + h.cosrot * (y - h.y0);
  const int n = (int)(yt / h.p.dy) + 1, m = (int)(xt / h.p.dx) + 1;
  if (n < 1 || n > h.p.nmax || m < 1 || m > h.p.mmax) return 0;
  const int32_t ic = h.dense2cmp[(size_t)m * h.p.ld + kGhostPad + n];
  return ic < 0 ? 0 : ic + 1;
}

size_t device_bytes_needed(const HostModel& h) {
  ScnDev d = h.p;
  int32_t *cmp = nullptr, *qmu = nullptr, *qmv = nullptr;
  Placer pl;
  place_model(h, d, cmp, qmu, qmv, pl, [](void*, const void*, size_t) {});
  return (pl.off + 255) & ~(size_t)255;
}

DeviceModel::DeviceModel(const HostModel& h) : h_(&h) {
  d_ = h.p;
  bytes_ = device_bytes_needed(h);
  check_cuda(cudaMalloc(&block_, bytes_), "cudaMalloc model");
  try {
    Placer pl;
    pl.base = static_cast<char*>(block_);
    place_model(h, d_, d_cmp_, d_qmap_u_, d_qmap_v_, pl, [](void* dst, const void* src, size_t n) {
      if (src)
        check_cuda(cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice), "upload");
      else
        check_cuda(cudaMemset(dst, 0, n), "cudaMemset");
    });
    StepState s{};
    s.t = h.t0;  // sfincs_lib.f90:279-282: t = t0, first min_dt = 1e-6
    s.tend = h.t0;
    s.min_dt = 1.0e-6f;
    s.dt = 1.0e-6f;
    s.itbndlast = s.itprcplast = s.itwndlast = s.itsrclast = 1;
    s.twindupd = (float)h.t0;  // sfincs_lib.f90:290
    s.steps_left = 0;
    float one_e_minus6 = 1.0e-6f;
    std::memcpy(&s.min_dt_bits, &one_e_minus6, 4);
    check_cuda(cudaMemcpy(d_.st, &s, sizeof(s), cudaMemcpyHostToDevice), "init step state");
  } catch (...) {
    cudaFree(block_);
    block_ = nullptr;
    throw;
  }
}

DeviceModel::~DeviceModel() {
  if (block_) cudaFree(block_);
}

// ============================================================================
// Runner
// ============================================================================
Runner::Runner(std::vector<DeviceModel*> models, int tile_m, cudaStream_t stream)
    : models_(std::move(models)), stream_(stream), own_stream_(stream == nullptr) {
  if (models_.empty()) throw std::runtime_error("Runner needs at least one model");
  if (tile_m != 8) throw std::runtime_error("only 32x8 cell tiles are built into this library");
  subgrid_ = models_[0]->host().p.subgrid;
  qt_ = models_[0]->host().p.quadtree;
  std::vector<ScnDev> scns;
  std::vector<Tile> tiles;
  for (size_t i = 0; i < models_.size(); i++) {
    const HostModel& h = models_[i]->host();
    if (h.p.subgrid != subgrid_) throw std::runtime_error("an ensemble must be all-subgrid or all-regular");
    if (h.p.quadtree != qt_) throw std::runtime_error("an ensemble must be all-quadtree or all-regular-grid");
    if (h.p.nsrc > 0 || h.p.ndrn > 0) any_src_ = 1;
    if (h.p.nstruc > 0) any_struc_ = 1;
    if (h.p.wind_field || h.p.patmos) met_ = 1;
    if (h.p.geo) geo_ = 1;
    if (h.p.inftype >= 2 || h.p.store_cumprcp || h.p.prcp_field || h.p.store_vmax || h.p.store_qmax ||
        h.p.store_twet || h.p.store_tzsmax || h.need_qinfmap)
      ext_ = 1;
    if (h.p.meteo3d) {
      any_meteo_ = 1;
      meteo_cells_ = std::max(meteo_cells_, (int)h.np);
    }
    bnd_blocks_ = std::max(bnd_blocks_, (h.p.nkcuv2 + h.p.nneu + 127) / 128);
    scns.push_back(models_[i]->dev());
    if (!qt_)
      for (const int2& t : h.tiles) tiles.push_back(Tile{(int)i, t.x, t.y, 0});
  }
  if (qt_) {
    // quadtree work lists: 256-wide chunks of uv points, combined points and cells
    auto chunks = [&](auto count_of) {
      int n = 0;
      for (size_t i = 0; i < models_.size(); i++) {
        const long long cnt = count_of(models_[i]->host());
        for (long long f0 = 0; f0 < cnt; f0 += 256, n++)
          tiles.push_back(Tile{(int)i, (int)f0, (int)std::min<long long>(256, cnt - f0), 0});
      }
      return n;
    };
    nqf_ = chunks([](const HostModel& h) { return h.npuv; });
    nqcuv_ = chunks([](const HostModel& h) { return (long long)h.p.ncuv; });
    nqc_ = chunks([](const HostModel& h) { return h.np; });
  }
  ntiles_ = (int)tiles.size();
  check_cuda(cudaMalloc(&d_scns_, scns.size() * sizeof(ScnDev)), "cudaMalloc scns");
  check_cuda(cudaMemcpy(d_scns_, scns.data(), scns.size() * sizeof(ScnDev), cudaMemcpyHostToDevice), "scns");
  if (ntiles_ > 0) {
    check_cuda(cudaMalloc(&d_tiles_, tiles.size() * sizeof(Tile)), "cudaMalloc tiles");
    check_cuda(cudaMemcpy(d_tiles_, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice), "tiles");
  }
  if (own_stream_) check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  if (const char* v = std::getenv("SFG_MOMENTUM_VARIANT")) {
    const int x = std::atoi(v);
    variant_ = (x >= 2 && x <= 5) ? x : 5;
  }
  if (geo_ && variant_ >= 4) variant_ = 2;  // the staged tile kernels assume one spacing per scenario
  if (!qt_) {
    // TMA tensor maps (one set per model) and persistent grid sizes
    std::vector<MapSet> maps;
    for (auto* m : models_) maps.push_back(build_map_set(m->dev()));
    check_cuda(cudaMalloc(&d_maps_, maps.size() * sizeof(MapSet)), "cudaMalloc maps");
    check_cuda(cudaMemcpy(d_maps_, maps.data(), maps.size() * sizeof(MapSet), cudaMemcpyHostToDevice), "maps");
    configure_grids();
  }
  check_cuda(cudaMallocHost(&h_states_, models_.size() * sizeof(StepState)), "pinned states");
  check_cuda(cudaMallocHost(&h_ctl_, models_.size() * sizeof(RunCtl)), "pinned run targets");
}

// Persistent grids of the TMA kernels: resident CTAs per SM x SM count, capped
// by the number of tiles.
void Runner::configure_grids() {
  if (qt_) return;  // quadtree kernels launch one CTA per work chunk
  int dev = 0, nsm = 0, nb_m = 0, nb_c = 0;
  check_cuda(cudaGetDevice(&dev), "device");
  check_cuda(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "sm count");
  const void* mfn = momentum_tma_fn(subgrid_, variant_ + (met_ ? 10 : 0), one() != nullptr);
  check_cuda(cudaFuncSetAttribute(mfn, cudaFuncAttributeMaxDynamicSharedMemorySize, momentum_tma_smem(variant_, subgrid_)),
             "momentum shared memory");
  check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb_m, mfn, 256, momentum_tma_smem(variant_, subgrid_)), "occupancy");
  check_cuda(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb_c, continuity_tma_fn(subgrid_, one() != nullptr, ext_ != 0), 256, continuity_tma_smem()),
      "occupancy");
  mom_grid_ = std::max(1, std::min(ntiles_, std::max(nb_m, 1) * nsm));
  con_grid_ = std::max(1, std::min(ntiles_, std::max(nb_c, 1) * nsm));
}

Runner::~Runner() {
  if (graph_) cudaGraphExecDestroy(graph_);
  if (d_maps_) cudaFree(d_maps_);
  if (stream_ && own_stream_) cudaStreamDestroy(stream_);
  if (d_scns_) cudaFree(d_scns_);
  if (d_tiles_) cudaFree(d_tiles_);
  if (h_states_) cudaFreeHost(h_states_);
  if (h_ctl_) cudaFreeHost(h_ctl_);
}

void Runner::launch_momentum_any() {
  if (qt_) {
    launch_qt_momentum(d_scns_, d_tiles_, nqf_, subgrid_, met_ != 0, stream_);
    launch_qt_cuv(d_scns_, d_tiles_ + nqf_, nqcuv_, stream_);
  } else if (tma()) {
    launch_momentum_tma(d_scns_, d_maps_, d_tiles_, ntiles_, subgrid_, variant_ + (met_ ? 10 : 0), mom_grid_, stream_,
                        one());
  } else {
    launch_momentum(d_scns_, d_tiles_, ntiles_, subgrid_, variant_, stream_);
  }
}

void Runner::launch_continuity_any() {
  if (qt_)
    launch_qt_continuity(d_scns_, d_tiles_ + nqf_ + nqcuv_, nqc_, subgrid_, ext_ != 0, stream_);
  else if (tma())
    launch_continuity_tma(d_scns_, d_maps_, d_tiles_, ntiles_, subgrid_, con_grid_, stream_, one(), ext_ != 0);
  else
    launch_continuity(d_scns_, d_tiles_, ntiles_, subgrid_, stream_);
}

void Runner::launch_one() {
  if (any_meteo_) launch_meteo_window(d_scns_, nscn(), meteo_cells_, stream_);
  launch_step_bnd(d_scns_, nscn(), bnd_blocks_, stream_, one());
  launch_momentum_any();
  if (any_struc_) launch_structures(d_scns_, nscn(), stream_);
  if (any_src_) launch_sources(d_scns_, nscn(), stream_);
  launch_continuity_any();
}

void Runner::build_graph(int chunk) {
  if (graph_ && graph_chunk_ == chunk) return;
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  cudaGraph_t g;
  check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
  for (int i = 0; i < chunk; i++) launch_one();
  check_cuda(cudaStreamEndCapture(stream_, &g), "end capture");
  check_cuda(cudaGraphInstantiate(&graph_, g, 0), "graph instantiate");
  cudaGraphDestroy(g);
  graph_chunk_ = chunk;
}

void Runner::refresh_params() {
  // single-model launches carry the parameters by value: re-capture the graph
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  std::vector<ScnDev> scns;
  for (auto* m : models_) scns.push_back(m->dev());
  check_cuda(cudaMemcpyAsync(d_scns_, scns.data(), scns.size() * sizeof(ScnDev), cudaMemcpyHostToDevice, stream_),
             "refresh params");
  sync();
}

void Runner::issue(int nsteps) {
  // whole chunks as CUDA-graph replays, the remainder as direct launches
  const int chunk = 32;
  if (nsteps >= chunk) {
    build_graph(chunk);
    for (int i = 0; i < nsteps / chunk; i++) check_cuda(cudaGraphLaunch(graph_, stream_), "graph launch");
  }
  for (int i = 0; i < nsteps % chunk; i++) launch_one();
}

std::vector<double> Runner::time_kernels(int nsteps) {
  std::vector<cudaEvent_t> ev(5);
  for (auto& e : ev) check_cuda(cudaEventCreate(&e), "event");
  std::vector<double> acc(4, 0.0);
  for (int i = 0; i < nsteps; i++) {
    check_cuda(cudaEventRecord(ev[0], stream_), "record");
    if (any_meteo_) launch_meteo_window(d_scns_, nscn(), meteo_cells_, stream_);
    launch_step_bnd(d_scns_, nscn(), bnd_blocks_, stream_, one());
    check_cuda(cudaEventRecord(ev[1], stream_), "record");
    launch_momentum_any();
    check_cuda(cudaEventRecord(ev[2], stream_), "record");
    if (any_struc_) launch_structures(d_scns_, nscn(), stream_);
    if (any_src_) launch_sources(d_scns_, nscn(), stream_);
    check_cuda(cudaEventRecord(ev[3], stream_), "record");
    launch_continuity_any();
    check_cuda(cudaEventRecord(ev[4], stream_), "record");
    check_cuda(cudaEventSynchronize(ev[4]), "event sync");
    for (int k = 0; k < 4; k++) {
      float ms = 0.0f;
      check_cuda(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]), "elapsed");
      acc[k] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (auto& a : acc) a /= std::max(nsteps, 1);
  return acc;
}

void Runner::sync() { check_cuda(cudaStreamSynchronize(stream_), "stream sync"); }

StepState Runner::read_state(int i) {
  check_cuda(cudaMemcpyAsync(&h_states_[i], models_[i]->state(), sizeof(StepState), cudaMemcpyDeviceToHost, stream_),
             "read state");
  sync();
  return h_states_[i];
}

void Runner::step_once(cudaEvent_t continuity_after) {
  // run targets from pinned memory (no pageable round trip); the step is then
  // stream-ordered before whatever the caller queues next (e.g. the zs refresh)
  for (size_t i = 0; i < models_.size(); i++) {
    h_ctl_[i].tend = models_[i]->host().t1;
    h_ctl_[i].steps_left = 1;
    check_cuda(cudaMemcpyAsync(&models_[i]->state()->tend, &h_ctl_[i].tend, sizeof(double), cudaMemcpyHostToDevice,
                               stream_),
               "tend");
    check_cuda(cudaMemcpyAsync(&models_[i]->state()->steps_left, &h_ctl_[i].steps_left, sizeof(int),
                               cudaMemcpyHostToDevice, stream_),
               "steps");
  }
  if (continuity_after) {
    if (any_meteo_) launch_meteo_window(d_scns_, nscn(), meteo_cells_, stream_);
    launch_step_bnd(d_scns_, nscn(), bnd_blocks_, stream_, one());
    launch_momentum_any();
    if (any_struc_) launch_structures(d_scns_, nscn(), stream_);
    if (any_src_) launch_sources(d_scns_, nscn(), stream_);
    check_cuda(cudaStreamWaitEvent(stream_, continuity_after, 0), "wait for the source terms");
    launch_continuity_any();
  } else {
    issue(1);
  }
  check_cuda(cudaGetLastError(), "step launch");
}

// Autotuner: times one chunk of real steps with each kernel variant on this
// runner's own models and keeps the fastest.  Every variant computes bitwise
// the same states (the GPU tests check it), so the choice never changes a
// result, and the tuning steps are part of the run.  Only meaningful while
// the models still have steps to take; returns the chosen variant.
int Runner::autotune(int chunk) {
  if (qt_ || geo_) return variant_;  // one quadtree kernel path; geographic grids on the per-thread kernels
  static const int kCandidates[] = {5, 4, 2};
  cudaEvent_t e0, e1;
  check_cuda(cudaEventCreate(&e0), "event");
  check_cuda(cudaEventCreate(&e1), "event");
  int best = variant_;
  float best_ms = 0.0f;
  tune_ms_.clear();
  for (int v : kCandidates) {
    set_variant(v);
    build_graph(chunk);
    check_cuda(cudaEventRecord(e0, stream_), "record");
    check_cuda(cudaGraphLaunch(graph_, stream_), "graph launch");
    check_cuda(cudaEventRecord(e1, stream_), "record");
    check_cuda(cudaEventSynchronize(e1), "event sync");
    float ms = 0.0f;
    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    tune_ms_.push_back({v, ms});
    if (best_ms == 0.0f || ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  set_variant(best);
  tuned_ = true;
  return best;
}

void Runner::run(const std::vector<double>& tend, long long max_steps, int chunk) {
  if (tend.size() != models_.size()) throw std::runtime_error("one target time per model is required");
  std::vector<double> tend_h = tend;
  std::vector<int> left((size_t)nscn(), max_steps >= 0 ? (int)std::min<long long>(max_steps, 0x7fffffff) : -1);
  for (int i = 0; i < nscn(); i++) {
    check_cuda(cudaMemcpyAsync(&models_[i]->state()->tend, &tend_h[i], sizeof(double), cudaMemcpyHostToDevice, stream_),
               "tend");
    check_cuda(cudaMemcpyAsync(&models_[i]->state()->steps_left, &left[i], sizeof(int), cudaMemcpyHostToDevice,
                               stream_),
               "steps");
  }
  auto all_done = [&]() {
    for (int i = 0; i < nscn(); i++) {
      const StepState& s = h_states_[i];
      if (!(s.stop_pending || !(s.t < s.tend) || s.steps_left == 0 || s.fault)) return false;
    }
    return true;
  };
  auto read_states = [&]() {
    for (int i = 0; i < nscn(); i++)
      check_cuda(cudaMemcpyAsync(&h_states_[i], models_[i]->state(), sizeof(StepState), cudaMemcpyDeviceToHost,
                                 stream_),
                 "read state");
  };
  if (autotune_ && !tuned_) {
    autotune(chunk);
    read_states();
    sync();
    if (all_done()) return;
  }
  build_graph(chunk);
  // Two chunks in flight: chunk k+1 is queued before the host looks at the
  // states copied after chunk k, so the GPU never waits for the host.  Steps
  // queued past a model's end are no-ops on the device (k_step stops it).
  cudaEvent_t ready;
  check_cuda(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event");
  check_cuda(cudaGraphLaunch(graph_, stream_), "graph launch");
  for (;;) {
    read_states();
    check_cuda(cudaEventRecord(ready, stream_), "record");
    check_cuda(cudaGraphLaunch(graph_, stream_), "graph launch");
    check_cuda(cudaEventSynchronize(ready), "event sync");
    if (all_done()) break;
  }
  cudaEventDestroy(ready);
  sync();
}

}  // namespace sfg
