// Map, his and max output (sfincs_output.f90:8-296, sfincs_ncoutput.F90:
// 148-1590, sfincs_ncoutput_helpers.F90:123-771) and the observation points
// (sfincs_obspoints.f90:4-140).
#include "output.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "inputs.h"
#include "ncwrite.h"

namespace sfg {

void launch_gather_f32(const float* src, const int32_t* cmp, float* out, long long n, cudaStream_t s);
void launch_gather_f64(const double* src, const int32_t* cmp, double* out, long long n, cudaStream_t s);
void launch_fill_f32(float* a, float v, long long n, cudaStream_t s);

namespace {

constexpr float kFill = -99999.0f;  // FILL_VALUE of the netCDF files
constexpr int kFillInt = -999;

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("output: ") + what + ": " + cudaGetErrorString(e));
}

// date_to_iso8601 of "yyyymmdd HHMMSS"
std::string iso8601(const std::string& t) {
  if (t.size() < 15) return t;
  return t.substr(0, 4) + "-" + t.substr(4, 2) + "-" + t.substr(6, 2) + " " + t.substr(9, 2) + ":" + t.substr(11, 2) +
         ":" + t.substr(13, 2);
}

// Fortran unformatted sequential record: length, data, length.
void fortran_record(FILE* f, const void* data, size_t bytes) {
  const int32_t n = (int32_t)bytes;
  std::fwrite(&n, 4, 1, f);
  std::fwrite(data, 1, bytes, f);
  std::fwrite(&n, 4, 1, f);
  std::fflush(f);
}

// Slots (gathered fields) of an output event
enum {
  S_ZS, S_UMD, S_UMU, S_VND, S_VNU, S_INF, S_ZVOL,                    // map
  S_ZSMAX, S_VMAX, S_QMAX, S_TWET, S_TZSMAX, S_CUMP, S_CUMI,          // max
  H_ZS, H_UMD, H_UMU, H_VND, H_VNU, H_QINF, H_S,                      // his (obs points)
  H_CRSU, H_CRSV,                                                     // his (cross-section faces: u, v fluxes)
  H_QDRN,                                                             // his (drainage structures)
  H_RUG,                                                              // his (run-up gauge points: zs)
  NSLOT
};

}  // namespace

// read_obs_points: sfincs_obspoints.f90:4-140
// read_rug_file: sfincs_runup_gauges.f90:3-115.  Per gauge (name line,
// "nrows ncols", its begin and end points) the cells of the points every
// 0.2 finest cell widths from the begin point; a point outside the mesh is
// refused (the reference would read level 0 there).
static void read_runup_gauges(HostModel& h, const std::string& file) {
  h.out.rug.clear();
  if (file.compare(0, 4, "none") == 0) return;
  std::vector<std::string> names;
  const auto pls = read_polylines(h.dir + "/" + file, 0, &names);
  const float dxyr = h.p.quadtree ? std::min(h.qt_dxr.back(), h.qt_dyr.back()) : std::min(h.p.dx, h.p.dy);
  const float dxstep = 0.2f * dxyr;
  for (size_t k = 0; k < pls.size(); k++) {
    if (pls[k].size() != 2) throw std::runtime_error("run-up gauge '" + names[k] + "' must have exactly two points");
    const float x0 = pls[k][0].x, y0 = pls[k][0].y, rdx = pls[k][1].x - x0, rdy = pls[k][1].y - y0;
    const float rlen = std::sqrt(rdx * rdx + rdy * rdy);
    const int nrp = (int)(rlen / dxstep) + 1;
    RunupGauge g;
    g.name = names[k];
    for (int ip = 1; ip <= nrp; ip++) {
      const float x = x0 + (float)(ip - 1) * dxstep * rdx / rlen;
      const float y = y0 + (float)(ip - 1) * dxstep * rdy / rlen;
      const int nm = cell_index(h, (double)x, (double)y);
      if (nm <= 0) throw std::runtime_error("run-up gauge '" + names[k] + "' leaves the active mesh");
      g.cells.push_back(nm);
    }
    h.out.rug.push_back(std::move(g));
  }
}

void read_obs_points(HostModel& h) {
  const std::string file = [&] {
    for (const auto& kv : h.out.inp)
      if (kv.first == "obsfile") return kv.second;
    return std::string("none");
  }();
  read_runup_gauges(h, [&] {
    for (const auto& kv : h.out.inp)
      if (kv.first == "rugfile") return kv.second;
    return std::string("none");
  }());
  h.out.obs.clear();
  h.need_qinfmap = h.p.infiltration && h.p.inftype == 5 && h.out.dtmapout > 1.0e-6 && h.out.map_type == "net";
  if (file.compare(0, 4, "none") == 0) return;
  std::ifstream f(h.dir + "/" + file);
  if (!f) throw std::runtime_error("cannot open observation points file " + file);
  int n = 0;
  for (std::string line; std::getline(f, line);) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    n++;
    ObsPoint o;
    const size_t j1 = line.find('\''), jdq = line.find('"');
    if (j1 == std::string::npos && jdq == std::string::npos) {
      char b[32];
      std::snprintf(b, sizeof b, "station_%03d", n);
      o.name = b;
    } else {
      const char q = j1 != std::string::npos ? '\'' : '"';
      const size_t a = line.find(q);
      const size_t e = line.find(q, a + 1);
      o.name = line.substr(a + 1, e == std::string::npos ? std::string::npos : e - a - 1);
      o.name.erase(0, o.name.find_first_not_of(' '));
      o.name.erase(o.name.find_last_not_of(' ') + 1);
    }
    std::string nums = line;
    for (char& ch : nums)
      if (ch == ',' || ch == '\t') ch = ' ';
    std::istringstream ls(nums);
    double x = 0, y = 0;
    if (!(ls >> x >> y)) throw std::runtime_error("observation points file " + file + ": bad line '" + line + "'");
    o.x = (float)x;
    o.y = (float)y;
    o.nm = cell_index(h, o.x, o.y);
    if (o.nm > 0) {
      o.xg = h.z_xz[(size_t)o.nm - 1];
      o.yg = h.z_yz[(size_t)o.nm - 1];
      o.zb = h.p.subgrid ? h.zmin_cmp[(size_t)o.nm - 1] : h.zb_cmp[(size_t)o.nm - 1];
    }
    h.out.obs.push_back(o);
  }
  const OutputSpec& out = h.out;
  h.need_qinfmap = h.p.infiltration &&
                   ((out.dthisout > 1.0e-6 && !out.obs.empty() && out.his_type == "net") ||
                    (h.p.inftype == 5 && out.dtmapout > 1.0e-6 && out.map_type == "net"));
}

OutputWriter::OutputWriter(const HostModel& h, DeviceModel& d, cudaStream_t main) : h_(h), d_(d), main_(main) {
  const OutputSpec& o = h.out;
  const ScnDev& P = h.p;
  np_ = (size_t)h.np;
  nobs_ = o.obs.size();
  ncrs_ = o.crs.size();
  nrug_ = o.rug.size();
  for (const auto& g : o.rug) nrug_pts_ += g.cells.size();
  for (const auto& cs : o.crs) ncrs_faces_ += cs.faces.size();
  // which files (sfincs_output.f90:8-58)
  if (o.dtmapout > 1.0e-6) {
    tmapout = o.t0out;
    map_net_ = o.map_type == "net";
    map_bin_ = !map_net_;
  }
  if (o.dtmaxout > 1.0e-6) {
    tmaxout = o.t0out + o.dtmaxout;
    // netCDF: into the map file, which exists only with map output; binary: files of their own
    max_on_ = o.map_type == "net" ? map_net_ : true;
  }
  if (o.dthisout > 1.0e-6 && (nobs_ > 0 || ncrs_ > 0 || nrug_ > 0)) {
    thisout = (double)h.t0;
    his_net_ = o.his_type == "net";
    his_txt_ = !his_net_;
  }
  if (!map_net_ && !map_bin_ && !max_on_ && !his_net_ && !his_txt_) return;
  infstate_ = P.inftype == 3 ? 3 : P.inftype == 4 ? 4 : P.inftype == 5 ? 5 : 0;

  check(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking), "stream");
  check(cudaEventCreateWithFlags(&gathered_, cudaEventDisableTiming), "event");
  check(cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming), "event");
  // gather maps: per cell the storage index of its md, nd, mu, nu uv points
  // (regular grids: the cell's own faces and those of its left / lower
  // neighbours), then per observation point its cell and faces
  ndrn_ = (size_t)P.ndrn;
  std::vector<int32_t> maps(4 * np_ + 5 * std::max<size_t>(nobs_, 1) + std::max<size_t>(ncrs_faces_, 1) + ndrn_ + nrug_pts_,
                            0);
  for (size_t i = 0; i < np_; i++) {
    if (P.quadtree) {
      const int4 c = h.qcell[i];
      maps[i] = c.x, maps[np_ + i] = c.z, maps[2 * np_ + i] = c.y, maps[3 * np_ + i] = c.w;
    } else {
      const int32_t c = h.cmp_off[i];
      maps[i] = c - P.ld, maps[np_ + i] = c - 1, maps[2 * np_ + i] = c, maps[3 * np_ + i] = c;
    }
  }
  for (size_t k = 0; k < nobs_; k++) {
    const int nm = o.obs[k].nm;
    if (nm <= 0) continue;
    for (int j = 0; j < 4; j++) maps[4 * np_ + j * nobs_ + k] = maps[(size_t)j * np_ + (size_t)nm - 1];
    maps[4 * np_ + 4 * nobs_ + k] = h.cmp_off[(size_t)nm - 1];
  }
  {  // then per cross-section face its flux storage (dense face offset, or quadtree uv point)
    size_t j = 4 * np_ + 5 * std::max<size_t>(nobs_, 1);
    for (const auto& cs : o.crs)
      for (const auto& f : cs.faces) maps[j++] = (int32_t)f.face;
    // then per drainage structure its intake entry of the source rates
    j = 4 * np_ + 5 * std::max<size_t>(nobs_, 1) + std::max<size_t>(ncrs_faces_, 1);
    for (size_t k = 0; k < ndrn_; k++) maps[j++] = (int32_t)(P.nsrc + 2 * k);
    // then the cell of every run-up gauge point
    for (const auto& g : o.rug)
      for (int32_t nm : g.cells) maps[j++] = h.cmp_off[(size_t)nm - 1];
  }
  check(cudaMalloc(&d_maps_, maps.size() * 4), "maps");
  check(cudaMemcpy(d_maps_, maps.data(), maps.size() * 4, cudaMemcpyHostToDevice), "maps");
  // staging
  slots_.resize(NSLOT);
  auto want = [&](int k, size_t n, size_t es) {
    Slot& s = slots_[(size_t)k];
    s.n = n;
    s.esize = es;
    check(cudaMalloc(&s.dev, n * es), "staging");
    check(cudaMallocHost(&s.host, n * es), "pinned staging");
  };
  const bool map_any = map_net_ || map_bin_;
  if (map_any) want(S_ZS, np_, 4);
  if (map_net_ && o.store_velocity)
    for (int k : {S_UMD, S_UMU, S_VND, S_VNU}) want(k, np_, 4);
  if (map_net_ && infstate_) want(S_INF, np_, 4);
  if (map_any && P.subgrid && o.store_zvolume) want(S_ZVOL, np_, 8);
  if (max_on_) {
    want(S_ZSMAX, np_, 4);
    if (P.store_vmax) want(S_VMAX, np_, 4);
    if (P.store_qmax) want(S_QMAX, np_, 4);
    if (P.store_twet) want(S_TWET, np_, 4);
    if (P.store_tzsmax) want(S_TZSMAX, np_, 4);
    if (d.dev().cumprcp) want(S_CUMP, np_, 4), want(S_CUMI, np_, 4);
  }
  if (his_net_ || his_txt_) {
    want(H_ZS, nobs_, 4);
    if (his_net_ && o.store_velocity)
      for (int k : {H_UMD, H_UMU, H_VND, H_VNU}) want(k, nobs_, 4);
    if (his_net_ && P.infiltration && d.dev().qinfmap) want(H_QINF, nobs_, 4);
    if (his_net_ && (P.inftype == 3 || P.inftype == 4)) want(H_S, nobs_, 4);
    if (his_net_ && ndrn_ > 0) want(H_QDRN, ndrn_, 4);
    if (his_net_ && nrug_pts_ > 0) want(H_RUG, nrug_pts_, 4);
    if (ncrs_faces_ > 0) {
      want(H_CRSU, ncrs_faces_, 4);
      if (!P.quadtree) want(H_CRSV, ncrs_faces_, 4);
    }
  }
  // file layout of the cell fields: (n, m) rows of the regular grid, or every point of the quadtree file
  file_idx_.resize(np_);
  if (P.quadtree) {
    ncells_file_ = h.qt_n.size();
    for (size_t q = 0; q < ncells_file_; q++)
      if (h.qt_nm[q] > 0) file_idx_[(size_t)h.qt_nm[q] - 1] = q;
  } else {
    ncells_file_ = (size_t)P.nmax * P.mmax;
    for (size_t i = 0; i < np_; i++) file_idx_[i] = (size_t)(h.z_n[i] - 1) * P.mmax + (size_t)(h.z_m[i] - 1);
  }
  huthresh_ = P.huthresh;
  if (map_net_) open_map();
  if (map_bin_) {
    zs_dat_ = std::fopen((h.dir + "/zs.dat").c_str(), "wb");
    if (!zs_dat_) throw std::runtime_error("cannot create zs.dat");
    if (P.subgrid && o.store_zvolume) zvol_dat_ = std::fopen((h.dir + "/z_volume.dat").c_str(), "wb");
  }
  if (max_on_ && !map_net_) open_max_bin();
  if (his_net_) open_his();
  if (his_txt_) {  // open_his_output: fresh text files
    std::remove((h.dir + "/zst.txt").c_str());
    if (P.precip) std::remove((h.dir + "/prcp.txt").c_str());
    if (ncrs_ > 0) std::remove((h.dir + "/qt.txt").c_str());
  }
  worker_ = std::thread([this] { run_worker(); });
}

OutputWriter::~OutputWriter() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  if (worker_.joinable()) worker_.join();
  for (Slot& s : slots_) {
    if (s.dev) cudaFree(s.dev);
    if (s.host) cudaFreeHost(s.host);
  }
  if (d_maps_) cudaFree(d_maps_);
  if (gathered_) cudaEventDestroy(gathered_);
  if (copied_) cudaEventDestroy(copied_);
  if (copy_) cudaStreamDestroy(copy_);
  for (FILE* f : max_dat_)
    if (f) std::fclose(f);
  if (zs_dat_) std::fclose(zs_dat_);
  if (zvol_dat_) std::fclose(zvol_dat_);
}

void OutputWriter::run_worker() {
  for (;;) {
    std::function<void()> job;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || !jobs_.empty(); });
      if (jobs_.empty()) return;
      job = std::move(jobs_.front());
      jobs_.pop_front();
      busy_ = true;
    }
    try {
      job();
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lk(mu_);
      if (error_.empty()) error_ = e.what();
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      busy_ = false;
    }
    cv_.notify_all();
  }
}

void OutputWriter::post(std::function<void()> job) {
  {
    std::lock_guard<std::mutex> lk(mu_);
    jobs_.push_back(std::move(job));
  }
  cv_.notify_all();
}

void OutputWriter::drain() {
  std::unique_lock<std::mutex> lk(mu_);
  cv_.wait(lk, [&] { return jobs_.empty() && !busy_; });
  if (!error_.empty()) {
    const std::string e = error_;
    error_.clear();
    throw std::runtime_error("output: " + e);
  }
}

void OutputWriter::gather(int k, const void* src, const int32_t* map, bool f64) {
  Slot& s = slot(k);
  if (!s.dev || !src) return;
  if (f64)
    launch_gather_f64((const double*)src, map, (double*)s.dev, (long long)s.n, main_);
  else
    launch_gather_f32((const float*)src, map, (float*)s.dev, (long long)s.n, main_);
}

// ---------------------------------------------------------------------------
// file layouts
// ---------------------------------------------------------------------------
namespace {

// A float variable of the cell dimensions with the reference's attributes (ncdef_float_var)
int def_cell_float(NcWriter& nc, const std::string& name, const std::vector<int>& dims, const char* units,
                   const char* long_name, const char* std_name, bool quadtree, const char* cell_methods = nullptr) {
  const int v = nc.def_var(name, NcWriter::FLOAT, dims);
  nc.att_float(v, "_FillValue", kFill);
  nc.att_text(v, "units", units);
  if (std_name && *std_name) nc.att_text(v, "standard_name", std_name);
  nc.att_text(v, "long_name", long_name);
  if (!quadtree) nc.att_text(v, "coordinates", "x y");
  if (cell_methods) nc.att_text(v, "cell_methods", cell_methods);
  if (quadtree) {
    nc.att_text(v, "mesh", "mesh2d");
    nc.att_text(v, "location", "face");
  }
  return v;
}

void put_inp(NcWriter& nc, const OutputSpec& o) {
  const int v = nc.def_var("inp", NcWriter::INT, {});
  for (const auto& kv : o.inp) nc.att_text(v, kv.first, kv.second);
}

}  // namespace

// ncoutput_map_init: sfincs_ncoutput.F90:148-774
void OutputWriter::open_map() {
  const HostModel& h = h_;
  const ScnDev& P = h.p;
  const OutputSpec& o = h.out;
  const bool qt = P.quadtree;
  map_nc_ = std::make_unique<NcWriter>();
  NcWriter& nc = *map_nc_;
  const long long nq = qt ? (long long)h.qt_n.size() : 0;
  std::vector<int> sp;
  int d_node = -1, d_face = -1, d_fn = -1, d_n = -1, d_m = -1, d_cn = -1, d_cm = -1;
  if (qt) {
    d_node = nc.def_dim("nmesh2d_node", 4 * nq);
    d_face = nc.def_dim("nmesh2d_face", nq);
    d_fn = nc.def_dim("max_nmesh2d_face_nodes", 4);
    sp = {d_face};
  } else {
    d_n = nc.def_dim("n", P.nmax);
    d_m = nc.def_dim("m", P.mmax);
    d_cn = nc.def_dim("corner_n", P.nmax + 1);
    d_cm = nc.def_dim("corner_m", P.mmax + 1);
    sp = {d_n, d_m};
  }
  const int d_time = nc.def_dim("time", NcWriter::UNLIMITED);
  const long long ntmx = std::max(1LL, (long long)std::ceil((o.t1out - o.t0out) / o.dtmaxout));
  const int d_tmax = nc.def_dim("timemax", ntmx);
  const int d_run = nc.def_dim("runtime", 1);
  auto with = [&](int first) {
    std::vector<int> v{first};
    v.insert(v.end(), sp.begin(), sp.end());
    return v;
  };
  nc.att_text(NcWriter::GLOBAL, "Conventions", qt ? "CF-1.8 UGRID-1.0 Deltares-0.10" : "CF-1.8 SGRID-0.3");
  nc.att_text(NcWriter::GLOBAL, "Producer", "SFINCS B200 core");
  nc.att_text(NcWriter::GLOBAL, "title", "SFINCS map netcdf output");
  put_inp(nc, o);
  int v_nx = -1, v_ny = -1, v_fnodes = -1, v_fx = -1, v_fy = -1, v_x = -1, v_y = -1, v_cx = -1, v_cy = -1;
  if (qt) {
    const int v_mesh = nc.def_var("mesh2d", NcWriter::INT, {d_run});
    nc.att_text(v_mesh, "cf_role", "mesh_topology");
    nc.att_text(v_mesh, "long_name", "Topology data of 2D network");
    nc.att_int(v_mesh, "topology_dimension", {2});
    nc.att_text(v_mesh, "node_coordinates", "mesh2d_node_x mesh2d_node_y");
    nc.att_text(v_mesh, "node_dimension", "nmesh2d_node");
    nc.att_text(v_mesh, "max_face_nodes_dimension", "max_nmesh2d_face_nodes");
    nc.att_text(v_mesh, "face_node_connectivity", "mesh2d_face_nodes");
    nc.att_text(v_mesh, "face_dimension", "nmesh2d_face");
    nc.att_text(v_mesh, "face_coordinates", "mesh2d_face_x mesh2d_face_y");
    for (int a = 0; a < 2; a++) {
      const int v = nc.def_var(a == 0 ? "mesh2d_node_x" : "mesh2d_node_y", NcWriter::DOUBLE, {d_node});
      nc.att_text(v, "units", "m");
      nc.att_text(v, "standard_name", a == 0 ? "projection_x_coordinate" : "projection_y_coordinate");
      nc.att_text(v, "long_name", a == 0 ? "x-coordinate of mesh nodes" : "y-coordinate of mesh nodes");
      nc.att_text(v, "grid_mapping", "crs");
      nc.att_text(v, "mesh", "mesh2d");
      nc.att_text(v, "location", "node");
      (a == 0 ? v_nx : v_ny) = v;
    }
    v_fnodes = nc.def_var("mesh2d_face_nodes", NcWriter::INT, {d_face, d_fn});
    nc.att_text(v_fnodes, "cf_role", "face_node_connectivity");
    nc.att_text(v_fnodes, "mesh", "mesh2d");
    nc.att_text(v_fnodes, "location", "face");
    nc.att_text(v_fnodes, "long_name", "Mapping from every face to its corner nodes (counterclockwise)");
    nc.att_int(v_fnodes, "start_index", {1});
    nc.att_int(v_fnodes, "_FillValue", {-999});
    for (int a = 0; a < 2; a++) {
      const int v = nc.def_var(a == 0 ? "mesh2d_face_x" : "mesh2d_face_y", NcWriter::DOUBLE, {d_face});
      nc.att_text(v, "units", "m");
      nc.att_text(v, "standard_name", a == 0 ? "projection_x_coordinate" : "projection_y_coordinate");
      nc.att_text(v, "long_name",
                  a == 0 ? "Characteristic x-coordinate of mesh face" : "Characteristic y-coordinate of mesh face");
      nc.att_text(v, "grid_mapping", "crs");
      nc.att_text(v, "mesh", "mesh2d");
      nc.att_text(v, "location", "face");
      (a == 0 ? v_fx : v_fy) = v;
    }
  } else {
    const int v_grid = nc.def_var("sfincsgrid", NcWriter::INT, {});
    nc.att_text(v_grid, "cf_role", "grid_topology");
    nc.att_int(v_grid, "topology_dimension", {2});
    nc.att_text(v_grid, "node_dimensions", "n m");
    nc.att_text(v_grid, "face_dimensions", "n: m:");
    nc.att_text(v_grid, "corner_dimensions", "corner_n: corner_m:");
    nc.att_text(v_grid, "face_coordinates", "x y");
    nc.att_text(v_grid, "corner_coordinates", "corner_x corner_y");
    auto axis = [&](const char* name, bool x, std::vector<int> dims, const char* long_name) {
      const int v = nc.def_var(name, NcWriter::FLOAT, dims);
      nc.att_float(v, "_FillValue", kFill);
      nc.att_text(v, "units", P.geo ? "degrees" : "m");  // def_grid_axis_coord
      nc.att_text(v, "standard_name", P.geo ? (x ? "longitude" : "latitude")
                                            : (x ? "projection_x_coordinate" : "projection_y_coordinate"));
      nc.att_text(v, "long_name", long_name);
      nc.att_text(v, "grid_mapping", "crs");
      nc.att_text(v, "grid", "sfincsgrid");
      return v;
    };
    v_x = axis("x", true, {d_n, d_m}, "face_x");
    v_y = axis("y", false, {d_n, d_m}, "face_y");
    v_cx = axis("corner_x", true, {d_cn, d_cm}, "corner_x");
    v_cy = axis("corner_y", false, {d_cn, d_cm}, "corner_y");
  }
  const int v_crs = nc.def_var("crs", NcWriter::INT, {});
  nc.att_int(v_crs, "epsg", {o.epsg});
  nc.att_text(v_crs, "epsg_code", "EPSG:" + o.epsg_code);
  const int v_msk = nc.def_var("msk", NcWriter::INT, sp);
  nc.att_int(v_msk, "_FillValue", {kFillInt});
  nc.att_text(v_msk, "long_name", "Active cells mask");
  nc.att_text(v_msk, "description",
              "inactive=0, active=1, normal_boundary=2, outflow_boundary=3, wavemaker=4, downstream_boundary=5, "
              "neumann_boundary=6");
  nc.att_text(v_msk, "units", "-");
  if (!qt) nc.att_text(v_msk, "coordinates", "x y");
  nc.att_int(v_msk, "flag_values", {0, 1, 2, 3, 4, 5, 6});
  nc.att_text(v_msk, "flag_meanings",
              "inactive active normal_boundary outflow_boundary wavemaker downstream_boundary neumann_boundary");
  if (qt) {
    nc.att_text(v_msk, "mesh", "mesh2d");
    nc.att_text(v_msk, "location", "face");
  }
  int v_qinf = -1;
  if (P.infiltration && (P.inftype == 1 || P.inftype == 2 || P.inftype == 3)) {
    v_qinf = P.inftype == 1 ? def_cell_float(nc, "qinf", sp, "mm h-1", "infiltration rate - constant in time", "qinf", qt)
             : P.inftype == 2 ? def_cell_float(nc, "qinf", sp, "m", "moisture storage (S) capacity - Curve number", "S", qt)
                              : def_cell_float(nc, "qinf", sp, "m", "maximum moisture storage (Smax) capacity - Curve number",
                                               "Smax", qt);
  }
  const int v_zb = def_cell_float(nc, "zb", sp, "m", "Bed level above reference level", "altitude", qt);
  const std::string tunits = "seconds since " + iso8601(h.tref);
  const int v_time = nc.def_var("time", NcWriter::FLOAT, {d_time});
  nc.att_text(v_time, "units", tunits);
  nc.att_text(v_time, "standard_name", "time");
  nc.att_text(v_time, "long_name", "time_in_seconds_since_" + iso8601(h.tref));
  const int v_zs =
      def_cell_float(nc, "zs", with(d_time), "m", "Water level", "sea_surface_height_above_reference_level", qt);
  int v_h = -1, v_u = -1, v_v = -1, v_zvol = -1, v_inf = -1;
  if (!P.subgrid || o.store_hsubgrid) v_h = def_cell_float(nc, "h", with(d_time), "m", "Water depth", "water_depth", qt);
  if (o.store_velocity) {
    v_u = def_cell_float(nc, "u", with(d_time), "m s-1", "Flow velocity x-component", "eastward_sea_water_velocity", qt);
    v_v = def_cell_float(nc, "v", with(d_time), "m s-1", "Flow velocity y-component", "northward_sea_water_velocity", qt);
  }
  if (P.subgrid && o.store_zvolume)
    v_zvol = def_cell_float(nc, "subgrid_volume", with(d_time), "m3", "Subgrid volume in cell", "subgrid_volume_in_cell", qt);
  if (infstate_ == 3) v_inf = def_cell_float(nc, "Seff", with(d_time), "m", "current moisture storage (Se) capacity", "Se", qt);
  if (infstate_ == 4) v_inf = def_cell_float(nc, "sigma", with(d_time), "-", "maximum soil moisture deficit", "sigma", qt);
  if (infstate_ == 5) v_inf = def_cell_float(nc, "f", with(d_time), "mm h-1", "current infiltration capacity", "f", qt);
  // max variables (ncoutput_map_init :496-560), in the order write_max_files fills them
  max_vars_.clear();
  if (max_on_) {
    const int v_tm = nc.def_var("timemax", NcWriter::FLOAT, {d_tmax});
    nc.att_text(v_tm, "units", tunits);
    nc.att_text(v_tm, "standard_name", "time");
    nc.att_text(v_tm, "long_name", "time_in_seconds_since_" + iso8601(h.tref));
    max_vars_.push_back(v_tm);
    max_vars_.push_back(def_cell_float(nc, "zsmax", with(d_tmax), "m", "Maximum water level",
                                       "maximum_sea_surface_height_above_reference_level", qt));
    max_vars_.push_back(P.store_cumprcp ? def_cell_float(nc, "cumprcp", with(d_tmax), "m", "Cumulative precipitation depth",
                                                         "cumulative_precipitation_depth", qt, "time: sum")
                                        : -1);
    max_vars_.push_back(P.store_twet ? def_cell_float(nc, "tmax", with(d_tmax), "seconds", "Time cell was wet",
                                                      "duration_wet", qt, "time: sum")
                                     : -1);
    max_vars_.push_back(P.store_tzsmax ? def_cell_float(nc, "t_zsmax", with(d_tmax), tunits.c_str(), "time when zsmax occurs",
                                                        "t_zsmax", qt, "time: maximum")
                                       : -1);
    max_vars_.push_back((!P.subgrid || o.store_hsubgrid)
                            ? def_cell_float(nc, "hmax", with(d_tmax), "m", "Maximum water depth",
                                             "sea_floor_depth_below_sea_surface", qt, "time: maximum")
                            : -1);
    max_vars_.push_back(P.store_vmax ? def_cell_float(nc, "vmax", with(d_tmax), "m s-1", "Maximum flow velocity",
                                                      "maximum_flow_velocity", qt, "time: maximum")
                                     : -1);
    max_vars_.push_back(P.store_qmax ? def_cell_float(nc, "qmax", with(d_tmax), "m^2 s-1", "maximum_flux", "maximum_flux",
                                                      qt, "time: maximum")
                                     : -1);
    max_vars_.push_back((P.store_cumprcp && P.infiltration)
                            ? def_cell_float(nc, "cuminf", with(d_tmax), "m", "cumulative_infiltration_depth", "", qt,
                                             "time: sum")
                            : -1);
  }
  static const char* const runtime_vars[3][3] = {{"total_runtime", "s", "Total model runtime (s)"},
                                                  {"average_dt", "s", "Average model time step (s)"},
                                                  {"status", "-", "status of SFINCS simulation - 0 is no error"}};
  for (const auto& r : runtime_vars) {
    const int v = nc.def_var(r[0], NcWriter::FLOAT, {d_run});
    nc.att_float(v, "_FillValue", kFill);
    nc.att_text(v, "units", r[1]);
    nc.att_text(v, "long_name", r[2]);
  }
  // record / fixed ids used later, by name order: zs, h, u, v, zvol, inf, time
  rec_ids_ = {v_time, v_zs, v_h, v_u, v_v, v_zvol, v_inf};
  nc.create(h.dir + "/sfincs_map.nc");
  // static fields
  if (qt) {
    const long long nq2 = nq;
    std::vector<double> nx(4 * nq2), ny(4 * nq2), fx(nq2), fy(nq2);
    std::vector<int32_t> fnodes(4 * nq2);
    const float x0 = h.x0, y0 = h.y0, cr = h.cosrot, sr = h.sinrot;
    for (long long i = 0; i < nq2; i++) {
      const int n = h.qt_n[i], m = h.qt_m[i], L = h.qt_lev[i];
      const float dxx = h.qt_dxr[(size_t)L - 1], dyy = h.qt_dyr[(size_t)L - 1];
      const int cm[4] = {m - 1, m, m, m - 1}, cn[4] = {n - 1, n - 1, n, n};
      for (int c = 0; c < 4; c++) {
        nx[4 * i + c] = x0 + cr * (float)cm[c] * dxx - sr * (float)cn[c] * dyy;
        ny[4 * i + c] = y0 + sr * (float)cm[c] * dxx + cr * (float)cn[c] * dyy;
        fnodes[4 * i + c] = (int32_t)(4 * i + c + 1);
      }
      fx[i] = x0 + cr * ((float)m - 0.5f) * dxx - sr * ((float)n - 0.5f) * dyy;
      fy[i] = y0 + sr * ((float)m - 0.5f) * dxx + cr * ((float)n - 0.5f) * dyy;
    }
    nc.put(v_nx, nx.data(), nx.size());
    nc.put(v_ny, ny.data(), ny.size());
    nc.put(v_fnodes, fnodes.data(), fnodes.size());
    nc.put(v_fx, fx.data(), fx.size());
    nc.put(v_fy, fy.data(), fy.size());
  } else {
    const int nmax = P.nmax, mmax = P.mmax;
    std::vector<float> xz((size_t)nmax * mmax), yz(xz.size()), xg((size_t)(nmax + 1) * (mmax + 1)), yg(xg.size());
    const float x0 = h.x0, y0 = h.y0, cr = h.cosrot, sr = h.sinrot, dx = P.dx, dy = P.dy;
    for (int n = 1; n <= nmax; n++)
      for (int m = 1; m <= mmax; m++) {
        const size_t k = (size_t)(n - 1) * mmax + (m - 1);
        xz[k] = x0 + cr * (1.0f * ((float)m - 0.5f)) * dx - sr * (1.0f * ((float)n - 0.5f)) * dy;
        yz[k] = y0 + sr * (1.0f * ((float)m - 0.5f)) * dx + cr * (1.0f * ((float)n - 0.5f)) * dy;
      }
    for (int n = 1; n <= nmax + 1; n++)
      for (int m = 1; m <= mmax + 1; m++) {
        const size_t k = (size_t)(n - 1) * (mmax + 1) + (m - 1);
        xg[k] = x0 + cr * (1.0f * (float)(m - 1)) * dx - sr * (1.0f * (float)(n - 1)) * dy;
        yg[k] = y0 + sr * (1.0f * (float)(m - 1)) * dx + cr * (1.0f * (float)(n - 1)) * dy;
      }
    nc.put(v_x, xz.data(), xz.size());
    nc.put(v_y, yz.data(), yz.size());
    nc.put(v_cx, xg.data(), xg.size());
    nc.put(v_cy, yg.data(), yg.size());
  }
  const int32_t epsg = o.epsg;
  nc.put(v_crs, &epsg, 1);
  {
    std::vector<float> zb(np_);
    std::vector<int32_t> msk(np_);
    for (size_t i = 0; i < np_; i++) {
      zb[i] = P.subgrid ? h.zmin_cmp[i] : h.zb_cmp[i];
      msk[i] = h.kcs_cmp[i];
    }
    std::vector<float> bz = scatter(zb.data());
    nc.put(v_zb, bz.data(), bz.size());
    std::vector<int32_t> bm(cells_total(), 0);
    for (size_t i = 0; i < np_; i++) bm[file_index(i)] = msk[i];
    nc.put(v_msk, bm.data(), bm.size());
    if (v_qinf >= 0) {
      std::vector<float> q(np_);
      for (size_t i = 0; i < np_; i++) {
        const size_t c = (size_t)h.cmp_off[i];
        q[i] = P.inftype == 1 ? h.qinf[c] * 3.6e6f : h.inf_par[0][c];
      }
      std::vector<float> bq = scatter(q.data());
      nc.put(v_qinf, bq.data(), bq.size());
    }
  }
  nc.sync();
}

std::vector<float> OutputWriter::scatter(const float* v, const std::vector<uint8_t>* keep) const {
  std::vector<float> b(cells_total(), kFill);
  for (size_t i = 0; i < np_; i++)
    if (!keep || (*keep)[i]) b[file_index(i)] = v[i];
  return b;
}

// ncoutput_his_init: sfincs_ncoutput.F90:779-1131 (observation points)
void OutputWriter::open_his() {
  const HostModel& h = h_;
  const ScnDev& P = h.p;
  const OutputSpec& o = h.out;
  his_nc_ = std::make_unique<NcWriter>();
  NcWriter& nc = *his_nc_;
  const int d_time = nc.def_dim("time", NcWriter::UNLIMITED);
  const int d_st = nc.def_dim("stations", (long long)std::max<size_t>(nobs_, 1));  // 1 without points, as the reference
  const int d_crs = ncrs_ > 0 ? nc.def_dim("crosssections", (long long)ncrs_) : -1;
  const int d_drn = ndrn_ > 0 ? nc.def_dim("drainage", (long long)ndrn_) : -1;
  const int d_rug = nrug_ > 0 ? nc.def_dim("runup_gauges", (long long)nrug_) : -1;
  const int d_len = nc.def_dim("pointnamelength", 256);
  const int d_run = nc.def_dim("runtime", 1);
  nc.att_text(NcWriter::GLOBAL, "Conventions", "CF-1.8");
  nc.att_text(NcWriter::GLOBAL, "featureType", "timeSeries");
  nc.att_text(NcWriter::GLOBAL, "Producer", "SFINCS B200 core");
  nc.att_text(NcWriter::GLOBAL, "title", "SFINCS his point netcdf output");
  put_inp(nc, o);
  const char* pt_coord = "station_id station_name point_x point_y";
  const int v_id = nc.def_var("station_id", NcWriter::FLOAT, {d_st});
  const int v_name = nc.def_var("station_name", NcWriter::CHAR, {d_st, d_len});
  nc.att_text(v_name, "cf_role", "timeseries_id");
  const int v_crsname = ncrs_ > 0 ? nc.def_var("crosssection_name", NcWriter::CHAR, {d_crs, d_len}) : -1;
  const int v_rugname = nrug_ > 0 ? nc.def_var("runup_gauge_name", NcWriter::CHAR, {d_rug, d_len}) : -1;
  auto coord = [&](const char* name, bool x, const char* long_name) {
    const int v = nc.def_var(name, NcWriter::FLOAT, {d_st});
    nc.att_text(v, "units", P.geo ? "degrees" : "m");  // def_his_point_coord
    nc.att_text(v, "standard_name", P.geo ? (x ? "longitude" : "latitude")
                                          : (x ? "projection_x_coordinate" : "projection_y_coordinate"));
    nc.att_text(v, "long_name", long_name);
    nc.att_text(v, "grid_mapping", "crs");
    return v;
  };
  const int v_sx = coord("station_x", true, "original_x_coordinate_of_station");
  const int v_sy = coord("station_y", false, "original_y_coordinate_of_station");
  const int v_px = coord("point_x", true, "point_x");
  const int v_py = coord("point_y", false, "point_y");
  const int v_crs = nc.def_var("crs", NcWriter::INT, {});
  nc.att_int(v_crs, "epsg", {o.epsg});
  nc.att_text(v_crs, "epsg_code", "EPSG:" + o.epsg_code);
  auto pvar = [&](const char* name, std::vector<int> dims, const char* units, const char* long_name,
                  const char* std_name) {
    const int v = nc.def_var(name, NcWriter::FLOAT, dims);
    nc.att_float(v, "_FillValue", kFill);
    nc.att_text(v, "units", units);
    if (std_name) nc.att_text(v, "standard_name", std_name);
    nc.att_text(v, "long_name", long_name);
    nc.att_text(v, "coordinates", pt_coord);
    return v;
  };
  const int v_zb = pvar("point_zb", {d_st}, "m", "Bed level above reference level", "altitude");
  const int v_time = nc.def_var("time", NcWriter::FLOAT, {d_time});
  nc.att_text(v_time, "units", "seconds since " + iso8601(h.tref));
  nc.att_text(v_time, "standard_name", "time");
  nc.att_text(v_time, "long_name", "time_in_seconds_since_" + iso8601(h.tref));
  his_ids_.assign(12, -1);
  his_ids_[0] = v_time;
  his_ids_[1] = pvar("point_zs", {d_time, d_st}, "m", "Water level", "sea_surface_height_above_reference_level");
  if (!P.subgrid || o.store_hsubgrid) his_ids_[2] = pvar("point_h", {d_time, d_st}, "m", "Water depth", "depth");
  if (o.store_velocity) {
    his_ids_[3] = pvar("point_u", {d_time, d_st}, "m s-1", "Flow velocity x-component", "sea_water_x_velocity");
    his_ids_[4] = pvar("point_v", {d_time, d_st}, "m s-1", "Flow velocity y-component", "sea_water_y_velocity");
    his_ids_[5] = pvar("point_uvmag", {d_time, d_st}, "m s-1", "Flow velocity magnitude", "sea_water_velocity");
    his_ids_[6] = pvar("point_uvdir", {d_time, d_st}, "degrees", "Flow velocity bearing (deg)",
                       "sea_water_velocity_direction");
  }
  if (slot(H_QINF).dev) his_ids_[7] = pvar("point_qinf", {d_time, d_st}, "mm hr-1", "Infiltration rate", nullptr);
  if (P.inftype == 3) his_ids_[8] = pvar("point_S", {d_time, d_st}, "m", "current moisture storage (Se) capacity", nullptr);
  if (P.inftype == 4) his_ids_[8] = pvar("point_S", {d_time, d_st}, "m", "maximum soil moisture deficit", nullptr);
  if (ncrs_ > 0) {  // ncoutput_his_init (sfincs_ncoutput.F90:1033-1036)
    his_ids_[9] = pvar("crosssection_discharge", {d_time, d_crs}, "m3 s-1", "discharge", nullptr);
    nc.att_text(his_ids_[9], "coordinates", "crosssection_name");
  }
  if (nrug_ > 0) {  // (:1043-1046)
    his_ids_[11] = pvar("runup_gauge_zs", {d_time, d_rug}, "m", "run-up elevation", nullptr);
    nc.att_text(his_ids_[11], "coordinates", "runup_gauge_name");
  }
  if (ndrn_ > 0)  // (:1038-1041)
    his_ids_[10] = pvar("drainage_discharge", {d_time, d_drn}, "m3 s-1", "discharge through drainage structure", nullptr);
  pvar("total_runtime", {d_run}, "s", "Total model runtime (s)", nullptr);
  pvar("average_dt", {d_run}, "s", "Average model time step (s)", nullptr);
  pvar("status", {d_run}, "-", "status of SFINCS simulation - 0 is no error", nullptr);
  nc.create(h.dir + "/sfincs_his.nc");
  std::vector<float> id(nobs_), sx(nobs_), sy(nobs_), px(nobs_), py(nobs_), zb(nobs_);
  std::vector<char> names(nobs_ * 256, ' ');
  for (size_t k = 0; k < nobs_; k++) {
    const ObsPoint& p = o.obs[k];
    id[k] = (float)(k + 1);
    sx[k] = p.x, sy[k] = p.y, px[k] = p.xg, py[k] = p.yg, zb[k] = p.zb;
    std::memcpy(&names[k * 256], p.name.data(), std::min<size_t>(p.name.size(), 256));
  }
  nc.put(v_id, id.data(), nobs_);
  nc.put(v_name, names.data(), names.size());
  nc.put(v_sx, sx.data(), nobs_);
  nc.put(v_sy, sy.data(), nobs_);
  nc.put(v_px, px.data(), nobs_);
  nc.put(v_py, py.data(), nobs_);
  nc.put(v_zb, zb.data(), nobs_);
  if (ncrs_ > 0) {
    std::vector<char> cn(ncrs_ * 256, ' ');
    for (size_t k = 0; k < ncrs_; k++)
      std::memcpy(&cn[k * 256], o.crs[k].name.data(), std::min<size_t>(o.crs[k].name.size(), 256));
    nc.put(v_crsname, cn.data(), cn.size());
  }
  if (nrug_ > 0) {
    std::vector<char> rn(nrug_ * 256, ' ');
    for (size_t k = 0; k < nrug_; k++)
      std::memcpy(&rn[k * 256], o.rug[k].name.data(), std::min<size_t>(o.rug[k].name.size(), 256));
    nc.put(v_rugname, rn.data(), rn.size());
  }
  const int32_t epsg = o.epsg;
  nc.put(v_crs, &epsg, 1);
  nc.sync();
}

// open_max_output: sfincs_output.f90:315-350 (binary max files)
void OutputWriter::open_max_bin() {
  const ScnDev& P = h_.p;
  const ScnDev& D = d_.dev();
  auto open = [&](const char* name, bool on) {
    FILE* f = nullptr;
    if (on) {
      f = std::fopen((h_.dir + "/" + name).c_str(), "wb");
      if (!f) throw std::runtime_error(std::string("cannot create ") + name);
    }
    max_dat_.push_back(f);
  };
  open("zsmax.dat", true);
  open("velmax.dat", P.store_vmax);
  open("tmax.dat", P.store_twet);
  open("cumprcp.dat", D.cumprcp != nullptr);
  open("cuminf.dat", D.cuminf != nullptr && P.infiltration);
  open("qmax.dat", P.store_qmax);
  open("t_zsmax.dat", P.store_tzsmax);
}

void OutputWriter::write(bool map, bool max, bool his, double tout, int p) {
  const ScnDev& D = d_.dev();
  const HostModel& h = h_;
  // the max fields start again at every max output time, with or without a
  // file to write them to (sfincs_output.f90:197-230)
  auto reset_max = [&] {
    const long long NA = D.quadtree ? (long long)h.np : (long long)D.nalloc;
    launch_fill_f32(D.zsmax, -999.0f, NA, main_);
    if (D.vmax) launch_fill_f32(D.vmax, -999.0f, NA, main_);
    if (D.qmax) launch_fill_f32(D.qmax, -999.0f, NA, main_);
    if (D.twet) launch_fill_f32(D.twet, 0.0f, NA, main_);
    if (D.tzsmax) launch_fill_f32(D.tzsmax, -999.0f, NA, main_);
    check(cudaGetLastError(), "max reset");
  };
  const bool reset = max && D.zsmax;
  map = map && (map_net_ || map_bin_);
  max = max && max_on_;
  his = his && (his_net_ || his_txt_);
  if (!map && !max && !his) {
    if (reset) reset_max();
    return;
  }
  drain();  // the staging buffers of the previous output are free
  const int32_t* cmp = d_.d_cmp_off();
  const int32_t* m4 = d_maps_;
  const int32_t* om = d_maps_ + 4 * np_;
  const float* uvu = D.uu[p];
  const float* uvv = D.quadtree ? D.uu[p] : D.vv[p];
  std::vector<int> got;
  auto g = [&](int k, const void* src, const int32_t* map_, bool f64 = false) {
    if (!slot(k).dev || !src) return;
    gather(k, src, map_, f64);
    got.push_back(k);
  };
  if (map) {
    g(S_ZS, D.zs, cmp);
    g(S_UMD, uvu, m4);
    g(S_VND, uvv, m4 + np_);
    g(S_UMU, uvu, m4 + 2 * np_);
    g(S_VNU, uvv, m4 + 3 * np_);
    g(S_INF, infstate_ == 5 ? (const float*)D.qinfmap : (const float*)D.inf_st[0], cmp);
    g(S_ZVOL, D.zvol, cmp, true);
  }
  if (max) {
    g(S_ZSMAX, D.zsmax, cmp);
    g(S_VMAX, D.vmax, cmp);
    g(S_QMAX, D.qmax, cmp);
    g(S_TWET, D.twet, cmp);
    g(S_TZSMAX, D.tzsmax, cmp);
    g(S_CUMP, D.cumprcp, cmp);
    g(S_CUMI, D.cuminf, cmp);
  }
  if (reset) reset_max();
  if (his) {
    g(H_ZS, D.zs, om + 4 * nobs_);
    g(H_UMD, uvu, om);
    g(H_VND, uvv, om + nobs_);
    g(H_UMU, uvu, om + 2 * nobs_);
    g(H_VNU, uvv, om + 3 * nobs_);
    g(H_QINF, D.qinfmap, om + 4 * nobs_);
    g(H_S, D.inf_st[0], om + 4 * nobs_);
    const int32_t* oc = d_maps_ + 4 * np_ + 5 * std::max<size_t>(nobs_, 1);
    g(H_CRSU, D.qu[p], oc);
    g(H_CRSV, D.quadtree ? nullptr : D.qv[p], oc);
    g(H_QDRN, D.qtsrc, oc + std::max<size_t>(ncrs_faces_, 1));
    g(H_RUG, D.zs, oc + std::max<size_t>(ncrs_faces_, 1) + ndrn_);
  }
  check(cudaGetLastError(), "gather launch");
  check(cudaEventRecord(gathered_, main_), "record");
  check(cudaStreamWaitEvent(copy_, gathered_, 0), "wait");
  for (int k : got)
    check(cudaMemcpyAsync(slot(k).host, slot(k).dev, slot(k).n * slot(k).esize, cudaMemcpyDeviceToHost, copy_), "d2h");
  check(cudaEventRecord(copied_, copy_), "record");
  const int rmap = ntmapout - 1, rmax = ntmaxout - 1, rhis = nthisout - 1;
  post([this, map, max, his, tout, rmap, rmax, rhis] {
    check(cudaEventSynchronize(copied_), "output copies");
    if (map) write_map_files(tout, rmap);
    if (max) write_max_files(tout, rmax);
    if (his) write_his_files(tout, rhis);
  });
}

// ncoutput_update_map (sfincs_ncoutput.F90:1138-1271) / write_map_output (sfincs_output.f90:400-424)
void OutputWriter::write_map_files(double tout, int rec) {
  const HostModel& h = h_;
  const ScnDev& P = h.p;
  const float* zs = (const float*)slot(S_ZS).host;
  const float* zref = P.subgrid ? h.zmin_cmp.data() : h.zb_cmp.data();
  if (map_bin_) {
    std::vector<double> z8(zs, zs + np_);
    fortran_record(zs_dat_, z8.data(), np_ * 8);
    if (zvol_dat_) fortran_record(zvol_dat_, slot(S_ZVOL).host, np_ * 8);
    return;
  }
  NcWriter& nc = *map_nc_;
  const float t4 = (float)tout;
  nc.put_record(rec_ids_[0], rec, &t4, 1);
  std::vector<uint8_t> wet(np_);
  for (size_t i = 0; i < np_; i++) wet[i] = (zs[i] - zref[i]) > huthresh_;
  std::vector<float> b = scatter(zs, &wet);
  nc.put_record(rec_ids_[1], rec, b.data(), b.size());
  if (rec_ids_[2] >= 0) {  // h: every cell on regular grids, wet cells on quadtree meshes
    std::vector<float> dep(np_);
    for (size_t i = 0; i < np_; i++) dep[i] = zs[i] - zref[i];
    b = scatter(dep.data(), P.quadtree ? &wet : nullptr);
    nc.put_record(rec_ids_[2], rec, b.data(), b.size());
  }
  if (rec_ids_[3] >= 0) {  // compute_uv_at_cell_centers (sfincs_ncoutput_helpers.F90:800-823)
    const float* umd = (const float*)slot(S_UMD).host;
    const float* umu = (const float*)slot(S_UMU).host;
    const float* vnd = (const float*)slot(S_VND).host;
    const float* vnu = (const float*)slot(S_VNU).host;
    std::vector<float> u(np_), v(np_);
    for (size_t i = 0; i < np_; i++) {
      float uz = 0.0f, vz = 0.0f;
      uz = uz + 0.5f * umd[i];
      uz = uz + 0.5f * umu[i];
      vz = vz + 0.5f * vnd[i];
      vz = vz + 0.5f * vnu[i];
      u[i] = h.cosrot * uz - h.sinrot * vz;
      v[i] = h.sinrot * uz + h.cosrot * vz;
    }
    b = scatter(u.data());
    nc.put_record(rec_ids_[3], rec, b.data(), b.size());
    b = scatter(v.data());
    nc.put_record(rec_ids_[4], rec, b.data(), b.size());
  }
  if (rec_ids_[5] >= 0) {
    const double* zv = (const double*)slot(S_ZVOL).host;
    std::vector<float> z4(np_);
    for (size_t i = 0; i < np_; i++) z4[i] = (float)zv[i];
    b = scatter(z4.data());
    nc.put_record(rec_ids_[5], rec, b.data(), b.size());
  }
  if (rec_ids_[6] >= 0) {
    b = scatter((const float*)slot(S_INF).host);
    nc.put_record(rec_ids_[6], rec, b.data(), b.size());
  }
  nc.sync();
}

// ncoutput_update_max (sfincs_ncoutput.F90:1443-1533) / write_max_output (sfincs_output.f90:426-468)
void OutputWriter::write_max_files(double tout, int rec) {
  const HostModel& h = h_;
  const ScnDev& P = h.p;
  const float* zref = P.subgrid ? h.zmin_cmp.data() : h.zb_cmp.data();
  const float* zsmax = (const float*)slot(S_ZSMAX).host;
  auto hostp = [&](int k) { return slot(k).host ? (const float*)slot(k).host : nullptr; };
  if (!map_net_) {
    std::vector<float> z(zsmax, zsmax + np_);
    for (size_t i = 0; i < np_; i++)
      if (z[i] < zref[i] + huthresh_) z[i] = -999.0f;
    const float* src[7] = {z.data(), hostp(S_VMAX), hostp(S_TWET), hostp(S_CUMP), hostp(S_CUMI), hostp(S_QMAX),
                           hostp(S_TZSMAX)};
    for (size_t j = 0; j < max_dat_.size(); j++)
      if (max_dat_[j] && src[j]) fortran_record(max_dat_[j], src[j], np_ * 4);
    return;
  }
  NcWriter& nc = *map_nc_;
  const long long ntmx = (long long)std::max(1.0, std::ceil((h.out.t1out - h.out.t0out) / h.out.dtmaxout));
  if (rec >= ntmx) return;  // beyond the timemax dimension
  const float t4 = (float)tout;
  nc.put(max_vars_[0], &t4, 1, (size_t)rec);
  const size_t nc_cells = cells_total();
  auto put = [&](int var, const std::vector<float>& b) { nc.put(var, b.data(), nc_cells, (size_t)rec * nc_cells); };
  std::vector<uint8_t> wet(np_);
  for (size_t i = 0; i < np_; i++) wet[i] = (zsmax[i] - zref[i]) > huthresh_;
  put(max_vars_[1], scatter(zsmax, &wet));
  if (max_vars_[2] >= 0 && hostp(S_CUMP)) put(max_vars_[2], scatter(hostp(S_CUMP)));
  if (max_vars_[3] >= 0) put(max_vars_[3], scatter(hostp(S_TWET)));
  if (max_vars_[4] >= 0) {  // t_zsmax where it was reached (min_value 0)
    const float* tz = hostp(S_TZSMAX);
    std::vector<uint8_t> pos(np_);
    for (size_t i = 0; i < np_; i++) pos[i] = tz[i] > 0.0f;
    put(max_vars_[4], scatter(tz, &pos));
  }
  if (max_vars_[5] >= 0) {
    std::vector<float> dep(np_);
    for (size_t i = 0; i < np_; i++) dep[i] = zsmax[i] - zref[i];
    put(max_vars_[5], scatter(dep.data(), &wet));
  }
  if (max_vars_[6] >= 0) put(max_vars_[6], scatter(hostp(S_VMAX)));
  if (max_vars_[7] >= 0) put(max_vars_[7], scatter(hostp(S_QMAX)));
  if (max_vars_[8] >= 0 && hostp(S_CUMI)) put(max_vars_[8], scatter(hostp(S_CUMI)));
  nc.sync();
}

// ncoutput_update_his (sfincs_ncoutput.F90:1275-1436) / write_his_output (sfincs_output.f90:577-620)
// get_discharges_through_crosssections (sfincs_crosssections.f90:130-176):
// per cross-section, in uv-point order, q times the crossing sign times the
// face width, summed in real*4.
std::vector<float> OutputWriter::crs_discharges() {
  const float* qu = (const float*)slot(H_CRSU).host;
  const float* qv = (const float*)slot(H_CRSV).host;
  std::vector<float> qq(ncrs_, 0.0f);
  size_t j = 0;
  for (size_t k = 0; k < ncrs_; k++)
    for (const auto& f : h_.out.crs[k].faces) {
      const float q = (f.dir == 0 || !qv) ? qu[j] : qv[j];
      qq[k] = qq[k] + q * f.idir * f.width;
      j++;
    }
  return qq;
}

void OutputWriter::write_his_files(double tout, int rec) {
  const HostModel& h = h_;
  const ScnDev& P = h.p;
  const OutputSpec& o = h.out;
  const float* zs = (const float*)slot(H_ZS).host;
  if (his_txt_) {  // zst.txt: f12.1 then f9.3 per point
    FILE* f = std::fopen((h.dir + "/zst.txt").c_str(), "a");
    if (!f) throw std::runtime_error("cannot append to zst.txt");
    std::fprintf(f, "%12.1f", tout);
    for (size_t k = 0; k < nobs_; k++) std::fprintf(f, "%9.3f", o.obs[k].nm > 0 ? zs[k] : -999.0f);
    std::fprintf(f, "\n");
    std::fclose(f);
    if (ncrs_ > 0) {  // qt.txt: f12.1 then f12.3 per cross-section
      const std::vector<float> qq = crs_discharges();
      FILE* fq = std::fopen((h.dir + "/qt.txt").c_str(), "a");
      if (!fq) throw std::runtime_error("cannot append to qt.txt");
      std::fprintf(fq, "%12.1f", tout);
      for (float v : qq) std::fprintf(fq, "%12.3f", v);
      std::fprintf(fq, "\n");
      std::fclose(fq);
    }
    return;
  }
  NcWriter& nc = *his_nc_;
  const float t4 = (float)tout;
  nc.put_record(his_ids_[0], rec, &t4, 1);
  std::vector<float> z(nobs_, kFill), hh(nobs_, kFill);
  for (size_t k = 0; k < nobs_; k++) {
    const int nm = o.obs[k].nm;
    if (nm <= 0) continue;
    z[k] = zs[k];
    hh[k] = zs[k] - (P.subgrid ? h.zmin_cmp[(size_t)nm - 1] : h.zb_cmp[(size_t)nm - 1]);
  }
  nc.put_record(his_ids_[1], rec, z.data(), nobs_);
  if (his_ids_[2] >= 0) nc.put_record(his_ids_[2], rec, hh.data(), nobs_);
  if (his_ids_[3] >= 0) {  // compute_uv_at_obs_points (sfincs_ncoutput_helpers.F90:745-771)
    const float* umd = (const float*)slot(H_UMD).host;
    const float* umu = (const float*)slot(H_UMU).host;
    const float* vnd = (const float*)slot(H_VND).host;
    const float* vnu = (const float*)slot(H_VNU).host;
    std::vector<float> u(nobs_, kFill), v(nobs_, kFill), mag(nobs_, kFill), dir(nobs_, kFill);
    for (size_t k = 0; k < nobs_; k++) {
      if (o.obs[k].nm <= 0) continue;
      const float uz = 0.5f * (umd[k] + umu[k]), vz = 0.5f * (vnd[k] + vnu[k]);
      u[k] = h.cosrot * uz - h.sinrot * vz;
      v[k] = h.sinrot * uz + h.cosrot * vz;
      mag[k] = std::sqrt(u[k] * u[k] + v[k] * v[k]);
      dir[k] = std::atan2(v[k], u[k]) * 180.0f / P.pi;
    }
    nc.put_record(his_ids_[3], rec, u.data(), nobs_);
    nc.put_record(his_ids_[4], rec, v.data(), nobs_);
    nc.put_record(his_ids_[5], rec, mag.data(), nobs_);
    nc.put_record(his_ids_[6], rec, dir.data(), nobs_);
  }
  auto point = [&](int id, int k, float scale) {  // write_point_var
    if (id < 0 || !slot(k).host) return;
    const float* v = (const float*)slot(k).host;
    std::vector<float> b(nobs_, kFill);
    for (size_t j = 0; j < nobs_; j++)
      if (o.obs[j].nm > 0) b[j] = v[j] * scale;
    nc.put_record(id, rec, b.data(), nobs_);
  };
  point(his_ids_[7], H_QINF, 3600000.0f);
  point(his_ids_[8], H_S, 1.0f);
  if (his_ids_[9] >= 0) {
    const std::vector<float> qq = crs_discharges();
    nc.put_record(his_ids_[9], rec, qq.data(), ncrs_);
  }
  if (his_ids_[11] >= 0) {  // get_runup_levels (sfincs_runup_gauges.f90:117-150): the last point wetter than rugdepth
    const float* z = (const float*)slot(H_RUG).host;
    std::vector<float> zru(nrug_, -999.0f);
    size_t j = 0;
    for (size_t k = 0; k < nrug_; k++)
      for (int32_t nm : o.rug[k].cells) {
        const float zbt = P.subgrid ? h.zmin_cmp[(size_t)nm - 1] : h.zb_cmp[(size_t)nm - 1];
        if (z[j] > zbt + o.rugdepth) zru[k] = z[j];
        j++;
      }
    nc.put_record(his_ids_[11], rec, zru.data(), nrug_);
  }
  if (his_ids_[10] >= 0 && slot(H_QDRN).host)  // qtsrc of each structure's intake (sfincs_ncoutput.F90:1410-1421)
    nc.put_record(his_ids_[10], rec, (const float*)slot(H_QDRN).host, ndrn_);
  nc.sync();
}

// finalize_output (sfincs_output.f90:260-296) with ncoutput_map_finalize / ncoutput_his_finalize
void OutputWriter::finalize(double t, double t1, int parity, float average_dt, int status) {
  if (max_on_) {
    if (ntmaxout == 0) {
      ntmaxout = 1;
      write(false, true, false, t, parity);
    } else if (t < tmaxout) {
      ntmaxout++;
      write(false, true, false, t1, parity);
    }
  }
  drain();
  const float st = (float)status;
  for (NcWriter* nc : {map_nc_.get(), his_nc_.get()}) {
    if (!nc) continue;
    nc->put(nc->var_id("average_dt"), &average_dt, 1);
    nc->put(nc->var_id("status"), &st, 1);
    nc->close();
  }
  for (FILE*& f : max_dat_)
    if (f) std::fclose(f), f = nullptr;
  if (zs_dat_) std::fclose(zs_dat_), zs_dat_ = nullptr;
  if (zvol_dat_) std::fclose(zvol_dat_), zvol_dat_ = nullptr;
}

}  // namespace sfg
