// Host side of the B200 SFINCS core: model loading (reference input files ->
// dense device layout), device residency, and the step runner (single model or
// an ensemble of uneven models advanced by the same launches).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "../sfg_device.h"

namespace sfg {

// One gridded meteo quantity as read from its ASCII file(s): nt records of
// nrows x ncols values, first row at the top; v[1] is the second wind component.
struct MeteoGridHost {
  int nt = 0, nrows = 0, ncols = 0;
  float x_ll = 0, y_ll = 0, dx = 0, dy = 0;
  std::vector<float> times, v[2];
};
// Reads an amu / amv / amp / ampr file into g (q: 0 first quantity, 1 second wind component).
void read_meteo_grid(const std::string& file, const std::string& tref, MeteoGridHost& g, int q);
// Seconds after tref of a meteo file's "TIME = <v> <unit> since <date>" line.
float meteo_time(const std::string& line, const std::string& tref);
// A spiderweb file as read: nt records of nrows x ncols polar values, the
// wind already in components, the pressure drop, the rain (zeros without a
// fourth quantity), the eye track.
struct SpwHost {
  int nt = 0, nrows = 0, ncols = 0, nquant = 0;
  bool precip = false;
  float radius = 0;
  std::vector<float> times, xe, ye, wu, wv, pdrp, prcp;
};
// Reads an ASCII spiderweb file (use_precip: usespwprecip).
void read_spw_file(const std::string& file, const std::string& tref, bool use_precip, SpwHost& s);

// An observation point of the obsfile (sfincs_obspoints.f90:4-140): its
// name and position, and the cell it falls in (1-based, 0 outside) with that
// cell's centre and bed level (-999 outside).
struct ObsPoint {
  std::string name;
  float x = 0, y = 0, xg = -999.0f, yg = -999.0f, zb = -999.0f;
  int nm = 0;
};
// Output settings (sfincs_input.f90:61-87, 274-294, 441-540), times in seconds after tref.
// One cross-section (sfincs_crosssections.f90:8-127): the uv points its
// polyline crosses, in uv-point order, each with the sign of the crossing
// and the face width; face is the dense offset of the u or v face (regular
// grids) or the uv point (quadtree meshes).
struct CrsFace {
  int64_t face;
  int dir;       // 0: u face, 1: v face
  float idir;    // +1 or -1
  float width;   // dyrm of a u face, dxrm of a v face (m)
};
struct CrossSection {
  std::string name;
  std::vector<CrsFace> faces;
};

// One run-up gauge (sfincs_runup_gauges.f90:3-150): the cells (1-based) of
// the points every 0.2 finest cell widths along its segment.
struct RunupGauge {
  std::string name;
  std::vector<int32_t> cells;
};

struct OutputSpec {
  double t0out = 0, t1out = 0, dtmapout = 0, dthisout = 600, dtmaxout = 9999999;
  std::string map_type = "net", his_type = "net";  // net: netCDF; bin: Fortran records; his asc/bin: text
  bool store_velocity = false, store_hsubgrid = false, store_zvolume = false;
  int epsg = 0;
  std::string epsg_code;
  std::vector<ObsPoint> obs;
  std::string crsfile = "none";
  std::vector<CrossSection> crs;
  float rugdepth = 0.05f;
  std::vector<RunupGauge> rug;
  std::vector<std::pair<std::string, std::string>> inp;  // the sfincs.inp keys, for the files' 'inp' attributes
};

// Astronomic boundary constituents after the nodal correction at tref: per
// constituent its frequency (rad/s), per point and constituent the amplitude
// times the nodal factor and the phase less V0+u (rad, in [0, 2 pi)); the first
// constituent is A0 (frequency 0).
struct TideHost {
  int ncomp = 0;
  std::vector<std::string> names;
  std::vector<double> omega;       // [ncomp]
  std::vector<double> amp, phase;  // [nbnd][ncomp]
};
void read_bca_file(const std::string& file, const std::string& tref, int nbnd, TideHost& out);

// Everything read from a model directory and laid out densely on the host.
struct HostModel {
  std::string dir;
  ScnDev p{};  // scalar parameters (pointer fields unused on the host copy)
  // switches and inputs that stay on the host
  bool store_vmax = false, store_qmax = false, store_twet = false;
  double t0 = 0, t1 = 0;
  long long np = 0, npuv = 0;
  // dense static arrays
  std::vector<uint16_t> flags;
  std::vector<float> zb, zbmx_u, zbmx_v, gn2_u, gn2_v;
  std::vector<float2> sgz_u, sgz_v;
  std::vector<float4> sgw_u, sgw_v;
  std::vector<UvRec> rec_u, rec_v;
  std::vector<float> zz_min, zz_max, zz_volmax;
  std::vector<float2> zlev;
  std::vector<float> qinf;
  // dense initial state
  std::vector<float> zs, zsmax, zs0;
  std::vector<double> zvol;
  std::vector<uint8_t> vneg;
  // compact (reference nm order) <-> dense
  std::vector<int32_t> cmp_off;           // [np] dense offset of compact cell nm-1
  std::vector<int32_t> dense2cmp;         // [nalloc] compact index (0-based) or -1
  float x0 = 0, y0 = 0, cosrot = 1, sinrot = 0;
  std::vector<float> z_xz, z_yz, zb_cmp, zmin_cmp;  // compact, for the BMI data interface
  std::vector<int8_t> kcs_cmp;
  std::vector<int32_t> z_n, z_m;
  // boundary lists (reference order of the kcuv==2 faces)
  std::vector<BndFace> bfaces;
  std::vector<int2> neu;               // Neumann cell, interior cell
  std::vector<int32_t> gb_cmp;         // compact index of every boundary cell (diagnostics)
  // forcing series
  std::vector<float> t_bnd, zs_bnd;  // zs_bnd [ntbnd][nbnd]
  TideHost tide;                     // astronomic constituents of the boundary points (bca file)
  std::vector<float> tprcp, vprcp, twnd, wmag, wdir, cdval;
  std::vector<float> x73;            // hu**(7/3) table when h73table is on (sfincs_data.f90:858-881)
  MeteoGridHost mgh[3];              // gridded meteo: 0 wind (amu, amv), 1 pressure (amp), 2 rain (ampr)
  std::string amufile = "none", amvfile = "none", ampfile = "none", amprfile = "none";  // their files
  SpwHost spw;                       // spiderweb (nt == 0: none)
  std::string spwfile = "none";
  bool use_spw_precip = true;
  float spw_merge_frac = 0.5f, factor_spw_size = 1.0f;
  std::vector<float> spw_pabs;       // absolute pressure of the web
  float factor_wind = 1, factor_pres = 1, factor_prcp = 1;
  // infiltration models with state: parameters, state, event flag, cumulative sums (storage order)
  std::vector<float> inf_par[5], inf_st[5], cumprcp, cuminf;
  std::vector<uint8_t> inf_rain;
  std::vector<float> tsrc, qsrc;     // qsrc [ntsrc][nsrc]
  std::vector<int32_t> src_cell;
  std::vector<StrucFace> struc;       // weir faces
  std::vector<DrnDev> drn;            // drainage structures
  std::vector<float> q0u, q0v, uv0u, uv0v, uvmean0;  // initial fluxes from a restart file (else zero)
  std::vector<uint8_t> kf0u, kf0v;                   // initial wet history with a restart file
  // restart output (sfincs_output.f90:8-58, 657-733): next time, interval, the
  // reference face order and the reference boundary-face order (-1: lateral Neumann face)
  std::string tref;
  double trstout = 1.0e9, dtrstout = 0.0;
  std::vector<int64_t> face_off;
  std::vector<int8_t> face_dir;
  std::vector<int> kb_bface;
  long long n_kcs1 = 0;
  double area_total_kcs1 = 0;
  std::vector<int2> tiles;  // (n0, m0) of every 32 x 8 tile holding an active cell
  // ---- quadtree meshes (p.quadtree != 0): compact cells and uv points
  std::vector<FaceQ> qface;
  std::vector<int4> qcell;
  std::vector<int2> qcuv;
  std::vector<uint8_t> qlev;
  std::vector<float> zbmx_q, gn2_q;
  std::vector<int32_t> qmap_u, qmap_v;  // q index of each cell's right / upper uv point (BMI qx, qy)
  std::vector<float> cell_area;         // [np] m2
  std::vector<int64_t> qt_key;          // sorted keys (level, m, n) of the active cells, for point lookup
  std::vector<int32_t> qt_key_cell;     // compact cell of each key
  // every point of the quadtree file (active or not), for the map file's mesh
  std::vector<int32_t> qt_n, qt_m, qt_nm;  // qt_nm: 1-based active cell, 0 inactive
  std::vector<uint8_t> qt_lev;
  std::vector<float> qt_dxr, qt_dyr;       // cell size per level
  // output
  OutputSpec out;
  bool need_qinfmap = false;               // an output reads the step's infiltration rate per cell
  std::vector<float> geo_dxm, geo_dxminv, geo_area, geo_fcor;  // geographic grids: per dense cell
};

class InpFile;

// Keywords of sfincs.inp needed after parsing (file names, grid, derived values).
struct Keys {
  int mmax = 0, nmax = 0;
  float dx = 0, dy = 0, x0 = 0, y0 = 0, rotation = 0, cosrot = 1, sinrot = 0, t0 = 0, t1 = 0;
  float hmin_cfl = 0, dtmax = 0, uvmax = 0, nuviscdim = 0, manning = 0, manning_land = 0, manning_sea = 0,
        rghlevland = 0, qinf = 0, qinf_zmin = 0;
  bool viscosity = false, advection_mask = true, quadtree = false;
  std::string thdfile, weirfile, drnfile, rstfile;  // thin dams, weirs, drainage structures, restart (regular grids)
  std::string inifile;                              // binary initial water levels (real*4, cell order)
  std::string bdrfile;                              // downstream river points
  std::string bcafile;                              // astronomic boundary constituents (when use_bcafile)
  // infiltration parameter files (binary real*4, cell order)
  std::string scsfile, smaxfile, sefffile, ksfile, psifile, sigmafile, f0file, fcfile, kdfile;
  std::string qtrfile, depfile, mskfile, indexfile, sbgfile, manningfile, bndfile, bzsfile, srcfile, disfile,
      wndfile, qinffile, prcpfile;
};
Keys parse_keys(const InpFile& in, HostModel& h, bool bmi);
// Polylines of a .thd / .weir file: x, y and npars values per point.
struct PolyRow {
  float x, y, p[2];
};
std::vector<std::vector<PolyRow>> read_polylines(const std::string& file, int npars,
                                                  std::vector<std::string>* names = nullptr);
// The sign of a crossing: +1 when the uv point's direction (cell nm to nmu)
// lies within pi counter-clockwise of the polyline segment (sfincs_crosssections.f90:92-107).
float crossing_sign(float xnm, float ynm, float xnmu, float ynmu, float xa, float ya, float xb, float yb, float pi);
// The reference's segment crossing test (geometry.f90 cross / direction, FP32).
bool segments_cross(float p1x, float p1y, float p2x, float p2y, float q1x, float q1y, float q2x, float q2y);
// One line of a drainage structures file: intake and outfall points, type, parameters.
struct DrnLine {
  float xs, ys, xo, yo;
  int type;
  float p[6];
};
std::vector<DrnLine> read_drainage(const std::string& file);
// Projected length of segment a-b onto segment 1-2 (geometry.f90:215-297).
float projected_length(float x0a, float y0a, float x0b, float y0b, float x1, float y1, float x2, float y2);
void read_boundary_series(HostModel& h, const Keys& k, bool water_level_bnd, std::vector<float>& xb,
                          std::vector<float>& yb, int& nbnd);
void read_meteo_series(HostModel& h, const Keys& k, float rotation);
// Infiltration models with state (cna, cnb, gai, hor; sfincs_infiltration.f90:
// 8-600): per-cell parameters from the binary files, converted as the
// reference does, laid out at storage index store[i] of compact cell i
// (nstore entries); the cumulative sums when stored.  P.inftype must be set.
void load_infiltration_models(HostModel& h, const Keys& k, size_t nstore, const std::vector<int32_t>& store);
// A binary restart file (sfincs_initial_conditions.F90:183-268): flavour, zs,
// q (npuv + ncuv + 1, reference order) and uvmean, and the infiltration state
// of flavours 4-6 (cnb: scs_Se; gai: GA_sigma, GA_F; hor: rain_T1).
struct RestartData {
  int type = 0;
  std::vector<float> zs, q, uvmean;
  std::vector<float> inf[2];
};
RestartData read_restart(const std::string& file);
// The infiltration state of a flavour 4-6 restart into the model's state arrays.
void apply_restart_infiltration(HostModel& h, const RestartData& rst, const std::vector<int32_t>& store);
// Quadtree mesh (qtrfile): compact cells and uv points (host/qtmodel.cpp).
void load_quadtree(HostModel& h, const Keys& k);
// 1-based active cell of a quadtree mesh at point (x, y), 0 outside.
int quadtree_cell_index(const HostModel& h, double x, double y);
// 1-based active cell of either mesh at point (x, y), 0 outside (find_quadtree_cell).
int cell_index(const HostModel& h, double x, double y);
// The obsfile's points with their cells (sfincs_obspoints.f90:4-140), into h.out.obs.
void read_obs_points(HostModel& h);

// Reads <dir>/sfincs.inp and the files it names.  bmi mirrors the reference's
// BMI initialize() (use_qext on).  Throws std::runtime_error on bad input.
std::unique_ptr<HostModel> load_model(const std::string& dir, bool bmi);

// Device residency of one model: all arrays allocated once, state updated in place.
class DeviceModel {
 public:
  explicit DeviceModel(const HostModel& h);
  ~DeviceModel();
  DeviceModel(const DeviceModel&) = delete;
  DeviceModel& operator=(const DeviceModel&) = delete;
  const HostModel& host() const { return *h_; }
  ScnDev& dev() { return d_; }
  StepState* state() { return d_.st; }
  size_t bytes() const { return bytes_; }
  // compact (nm order) views
  int32_t* d_cmp_off() { return d_cmp_; }
  // q index of each cell's right / upper uv point (quadtree meshes; null otherwise)
  const int32_t* d_qmap_u() const { return d_qmap_u_; }
  // gather map of a per-cell face array: dir 0 = right (x) face, 1 = upper (y) face
  const int32_t* face_map(int dir) const {
    if (d_qmap_u_) return dir == 0 ? d_qmap_u_ : d_qmap_v_;
    return d_cmp_;
  }
  const int32_t* d_qmap_v() const { return d_qmap_v_; }

 private:
  const HostModel* h_;
  ScnDev d_{};
  void* block_ = nullptr;  // every device array of the model, one allocation
  int32_t* d_cmp_ = nullptr;
  int32_t *d_qmap_u_ = nullptr, *d_qmap_v_ = nullptr;
  size_t bytes_ = 0;
};

// Device bytes a DeviceModel of h will allocate (exact; no allocation made).
size_t device_bytes_needed(const HostModel& h);

// Advances one or more device models together.  Every launch covers all
// models; models whose time has reached their own target are skipped on the
// device (no host round trip per step).
class Runner {
 public:
  // stream: run on this stream (not owned); null: the runner creates its own.
  Runner(std::vector<DeviceModel*> models, int tile_m = 8, cudaStream_t stream = nullptr);
  ~Runner();
  // Run until every model reached its target time; at most max_steps steps
  // per model when max_steps >= 0.  Steps are issued in CUDA-graph chunks of
  // `chunk` steps; the host checks completion once per chunk.
  void run(const std::vector<double>& tend, long long max_steps, int chunk = 32);
  // Autotune the kernel variant on the next chunk of steps (see model.cpp).
  int autotune(int chunk = 32);
  void set_autotune(bool on) { autotune_ = on; }
  const std::vector<std::pair<int, float>>& tune_ms() const { return tune_ms_; }
  // One step exactly (reference update()); queued on the stream, not waited for.
  // continuity_after: an event the continuity kernel of the step waits for (an
  // update of its source terms still in flight on another stream), or null.
  void step_once(cudaEvent_t continuity_after = nullptr);
  void sync();
  cudaStream_t stream() const { return stream_; }
  StepState read_state(int i);
  // re-upload the scalar parameters of every model (after a host-side change)
  void refresh_params();
  const ScnDev* d_scns() const { return d_scns_; }
  int ntiles() const { return ntiles_; }
  int bnd_blocks() const { return bnd_blocks_; }
  // kernel variant (momentum occupancy target); SFG_MOMENTUM_VARIANT overrides the default
  void set_variant(int v) {
    variant_ = (geo_ && v >= 4) ? 2 : v;  // geographic grids run the per-thread kernels
    if (graph_) {
      cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
    }
    configure_grids();
  }
  int variant() const { return variant_; }
  // variants 4 and 5: TMA-staged kernels (momentum compiled for 3 / 4 CTAs/SM);
  // 2 and 3: per-thread-load kernels
  bool tma() const { return variant_ >= 4; }
  // the one model of a single-model runner (its parameters travel by value in
  // the launches), null for an ensemble
  const ScnDev* one() const { return models_.size() == 1 ? &models_[0]->dev() : nullptr; }
  // launch one step (all kernels) on the runner's stream
  void launch_one();
  int nscn() const { return (int)models_.size(); }
  // issue `nsteps` steps on the stream (no host sync); used for timing
  void issue(int nsteps);
  // Issue nsteps steps with CUDA events between the launches; returns the mean
  // duration (ms) of [step+boundary, momentum, sources, continuity] launches.
  std::vector<double> time_kernels(int nsteps);
  int launches_per_step() const { return 3 + any_src_ + any_struc_ + any_meteo_ + (qt_ && nqcuv_ > 0 ? 1 : 0); }

 private:
  void build_graph(int chunk);
  void configure_grids();
  void launch_momentum_any();
  void launch_continuity_any();
  std::vector<DeviceModel*> models_;
  ScnDev* d_scns_ = nullptr;
  Tile* d_tiles_ = nullptr;
  int ntiles_ = 0;
  int bnd_blocks_ = 0;
  int variant_ = 5;
  MapSet* d_maps_ = nullptr;  // TMA tensor maps, one set per model
  int mom_grid_ = 0, con_grid_ = 0;
  int subgrid_ = 0;
  int qt_ = 0;                       // quadtree models: face / combined-point / cell work lists in d_tiles_
  int nqf_ = 0, nqcuv_ = 0, nqc_ = 0;
  int any_src_ = 0, any_struc_ = 0;
  int any_meteo_ = 0, meteo_cells_ = 0;  // gridded meteo: the window kernel runs before each step kernel
  int met_ = 0;  // gridded wind or pressure: momentum runs its meteo instance (variant + 10)
  int ext_ = 0;  // continuity runs its extended instance (infiltration with state, sums, gridded rain, store variables)
  int geo_ = 0;  // a geographic grid: per-cell spacing, on the per-thread kernels (variants 2 and 3)
  cudaStream_t stream_ = nullptr;
  bool own_stream_ = true;
  cudaGraphExec_t graph_ = nullptr;
  int graph_chunk_ = 0;
  StepState* h_states_ = nullptr;  // pinned mirror of the step states
  struct RunCtl {
    double tend;
    int steps_left;
  };
  RunCtl* h_ctl_ = nullptr;  // pinned run targets of step_once()
  bool autotune_ = false, tuned_ = false;
  std::vector<std::pair<int, float>> tune_ms_;  // (variant, ms per chunk) of the last autotune
};

void launch_step(const ScnDev* d_scns, int nscn, int bnd_blocks, const Tile* d_tiles, int ntiles, int subgrid,
                 int any_src, int variant, cudaStream_t s);
void launch_step_bnd(const ScnDev* d_scns, int nscn, int bnd_blocks, cudaStream_t s, const ScnDev* one);
void launch_meteo_window(const ScnDev* d_scns, int nscn, int max_cells, cudaStream_t s);
void launch_momentum(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, int variant,
                     cudaStream_t s);
void launch_sources(const ScnDev* d_scns, int nscn, cudaStream_t s);
void launch_structures(const ScnDev* d_scns, int nscn, cudaStream_t s);
void launch_continuity(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, cudaStream_t s);

void check_cuda(cudaError_t e, const char* what);

MapSet build_map_set(const ScnDev& d);
int momentum_tma_smem(int form, int subgrid);
int continuity_tma_smem();
const void* momentum_tma_fn(int subgrid, int form, bool one);
const void* continuity_tma_fn(int subgrid, bool one, bool ext);
void launch_momentum_tma(const ScnDev* d_scns, const MapSet* d_maps, const Tile* d_tiles, int ntiles, int subgrid,
                         int form, int grid, cudaStream_t s, const ScnDev* one);
void launch_continuity_tma(const ScnDev* d_scns, const MapSet* d_maps, const Tile* d_tiles, int ntiles, int subgrid,
                           int grid, cudaStream_t s, const ScnDev* one, bool ext);
void launch_qt_momentum(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, bool met, cudaStream_t s);
void launch_qt_cuv(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, cudaStream_t s);
void launch_qt_continuity(const ScnDev* d_scns, const Tile* d_tiles, int ntiles, int subgrid, bool ext,
                          cudaStream_t s);

}  // namespace sfg
