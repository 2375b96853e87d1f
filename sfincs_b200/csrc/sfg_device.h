// Device-side data layout of the B200 SFINCS core.
//
// Regular (and regular-subgrid) meshes are stored DENSE: every array is a
// padded (mmax+2) x ld column-major grid with n (y) fastest, so that the
// reference's twelve explicit uv neighbour index arrays
// (sfincs_domain.f90:1007-1261) become implicit +-1 / +-ld offsets and every
// warp reads 32 consecutive cells.  Cell (n, m), 1-based as in the reference,
// sits at   off(n, m) = m*ld + 31 + n   (n = 0 and n = nmax+1, m = 0 and
// m = mmax+1 are inactive ghost cells; n = 1 lands on a 128-byte boundary).
// The u face at off(n,m) joins (n,m)-(n,m+1); the v face joins (n,m)-(n+1,m).
// Faces that do not exist in the reference keep q = uv = 0 forever, which is
// exactly the reference's "dummy" uv point npuv+ncuv+1.
//
// All kernels are written against a table of scenarios, so one launch can
// advance a single model (the BMI drop-in) or many uneven models (ensembles).
#pragma once
#include <cstdint>

namespace sfg {

constexpr int kGhostPad = 31;  // low padding so that n = 1 is 128-byte aligned
constexpr int kRecFull = 255;  // record-cache code of the full branch (zsu above the table)
constexpr int kMaxSubgridLevels = 254;  // level codes 1..nlev-1 stay below kRecFull

// Static per-cell flag bits (uint16_t).
enum : uint16_t {
  F_ACT = 1u << 0,     // cell exists (msk > 0)
  F_KCS1 = 1u << 1,    // kcs == 1: continuity update
  F_UACT = 1u << 2,    // u face exists and kcuv in {1,6}: momentum update
  F_VACT = 1u << 3,    // v face exists and kcuv in {1,6}
  F_UADV = 1u << 4,    // u face mask_adv == 1
  F_VADV = 1u << 5,    // v face mask_adv == 1
  F_CDN = 1u << 6,     // cell (n-1,m) exists  (u face u_ndm neighbour; else self)
  F_CUP = 1u << 7,     // cell (n+1,m) exists  (u face u_num neighbour; else self)
  F_CLF = 1u << 8,     // cell (n,m-1) exists  (v face u_ndm neighbour; else self)
  F_CRT = 1u << 9,     // cell (n,m+1) exists  (v face u_num neighbour; else self)
  F_UTH = 1u << 10,    // u face: kcuv(u_nmd)==1 and kcuv(u_nmu)==1 (theta smoothing)
  F_VTH = 1u << 11,    // v face: same
};

// Per-face wet history (uint8_t, one array per face direction, mutable):
// bit 0 = wet after the previous step (the reference's kfuv), bit 1 = wet the
// step before.  A face dry for two consecutive steps holds q = uv = 0 in both
// ping-pong buffers, so its (zero) writes are skipped.
// Wet history of a face: KF_WET wet at the previous step, KF_WET2 wet the step
// before (so the ping-pong buffer being written may hold a nonzero flux);
// KF_STALE: both buffers hold fluxes from a restart file.  For the buffer
// bookkeeping KF_STALE counts as wet at the previous step, for friction (the
// newly-wet formula) it does not.
enum : uint8_t { KF_WET = 1u, KF_WET2 = 2u, KF_STALE = 4u };

// One weir face (kcuv = 3, sfincs_structures.f90:38-381): the uv face with
// the dense offsets of its two cells, the crest level and discharge
// coefficient interpolated along the weir polyline, and the crossed length
// relative to the face width.
struct alignas(16) StrucFace {
  int face;      // dense offset of the face (the cell that owns it)
  int nm, nmu;   // dense offsets of the cells on either side
  int dir;       // 0: u face, 1: v face
  float height;  // crest level
  float cd;      // discharge coefficient
  float len;     // crossed length / face width
  int pad;
};

// One drainage structure (sfincs_discharges.f90:180-320): type 1 pump, 2
// culvert, 3 check valve, 4 gate controlled by the intake level, 5 gate
// controlled by time; the dense offsets of its intake and outfall cells.
struct alignas(16) DrnDev {
  int type;
  int cin, cout;    // intake (sink) and outfall (source) cells
  int pad;
  float p[6];       // pump: q; culvert / valve: coefficient; gates: width, sill, n, zmin|tclose, zmax|topen, closing time
  float distance;   // between the two cell centres
  float pad2;
};

// One water-level boundary face (kcuv == 2), packed so one thread reads it in
// three 16-byte loads.  The boundary cell's level is recomputed per face from
// the two nearest boundary points (sfincs_boundaries.f90:806-876).
struct alignas(16) BndFace {
  int face;      // dense offset of the face
  int nmb;       // dense offset of the boundary cell
  int nmi;       // dense offset of the interior cell
  int info;      // bit0: v face; bit1: ibuvdir = +1 (else -1); bit2: outflow cell (kcs 3); bit3: multiple bnd points;
                 // bit4: a weir on the face (kcuv 3: no boundary flux); bit5: downstream river cell (kcs 5)
  int i1, i2;    // nearest boundary points (0-based)
  float fac;     // weight of i1
  float zbuv;    // zbuv of the face (regular grids; sfincs_domain.f90:1692)
  float floor;   // zb or subgrid z_zmin of the boundary cell
  float zfix;    // fixed level of an outflow (kcs 3) cell (sfincs_domain.f90:1937-1948); river (kcs 5): the level
                 // difference dzs_bdr to the internal point (sfincs_boundaries.f90:250-263)
  float len;     // face length (m): dy for u faces, dx for v faces (per refinement level on a quadtree)
  int zsi;       // river (kcs 5): dense offset of the cell holding the internal point
};

// ---- quadtree layout ---------------------------------------------------------
// Cells and uv points are compact, in the reference's order (sfincs order:
// by level, then n fastest).  q/uv arrays hold npuv faces, then ncuv combined
// points (mean of the two fine faces at a refinement transition,
// sfincs_momentum.f90:757-779), then one dummy entry that stays 0.
constexpr int kMaxQtLevels = 8;
enum : uint32_t {
  QF_DIR = 1u,     // v face
  QF_ACT = 2u,     // kcuv 1 or 6: the momentum kernel updates the face
  QF_ADV = 4u,     // advection mask (sfincs_domain.f90:2147-2178)
  QF_TH = 8u,      // theta smoothing allowed: kcuv(u_nmd) == kcuv(u_nmu) == 1
  QF_TRANS = 16u,  // refinement transition face (uv_flags_type != 0)
};
struct alignas(16) FaceQ {
  int nm, nmu;                       // cells on either side (0-based)
  int u_nmd, u_nmu, u_ndm, u_num;    // uv neighbours (sfincs_domain.f90:1007-1261), 0-based q indices
  int v_ndm, v_nm, v_ndmu, v_nmu;
  uint32_t info;                     // QF_* bits; bits 8..11: refinement level - 1
  int pad;
};

// One subgrid uv lookup record: values at level k and the increment to k+1
// (computed with the same float subtraction the reference performs inline at
// sfincs_momentum.f90:376-378), so one 32-byte sector serves one lookup.
struct alignas(32) UvRec {
  float havg, dhavg, nrep, dnrep, pwet, dpwet, pad0, pad1;
};

// Per-scenario mutable step state (device memory).  Time is FP64.
struct alignas(16) StepState {
  double t;            // model time (s), reference sfincs_lib.f90:57 real*8
  double tend;         // end of the current update interval
  double bflux_vol;    // FP64 accumulated boundary inflow volume (m3)
  double rain_vol;     // FP64 accumulated rain depth (m); times the kcs==1 area gives the volume
  double src_vol;      // FP64 accumulated point-source volume (m3)
  unsigned int min_dt_bits;  // float bits; atomicMin target of the flux kernel
  float dt;            // current step (real*4)
  float min_dt;        // min_dt used for the current dt
  float ptmp;          // uniform rain for this step (m/s)
  float twu, twv;      // uniform wind stress for this step
  int nt;              // steps taken
  int run;             // 1 if the current step executes
  int parity;          // which q/uv buffer holds the latest values
  int error;           // 1 = instability stop (sfincs_lib.f90:634-648)
  int stop_pending;    // instability detected: t := t1 + 1 at the next step
  float tbfac;         // boundary time-interpolation factor of the current step
  int itb0, itb1;      // boundary time records of the current step (1-based)
  int steps_left;      // for single / bounded calls
  int itbndlast, itprcplast, itwndlast, itsrclast;
  int fault;           // nonzero: a bounded wait in a staged kernel gave up (its tile was skipped)
  float ga_hs;         // Green-Ampt: GA_head * GA_sigma of the model's last cell at the start of the step
  // gridded meteo update window (sfincs_lib.f90:493-503), real*4 like the reference
  float twindupd;      // next window start
  float meteo_t0, meteo_t1;
  int pad_m;
};

// One gridded meteo quantity on an equidistant grid (ASCII amu/amv, amp,
// ampr; sfincs_spiderweb.f90:135-230): nt records of nrows x ncols values,
// the first row at the top, as the file holds them.
struct MeteoGrid {
  int nt, nrows, ncols, pad;
  float x_ll, y_ll, dx, dy;
  const float* times;  // [nt] seconds after tref
  const float* v0;     // [nt][nrows][ncols]: amu, amp or ampr
  const float* v1;     // amv (wind only)
};

// A spiderweb: wind, pressure and rain on a polar grid around a moving
// cyclone eye (ASCII spw file, sfincs_spiderweb.f90:8-134, with the
// conversions of read_meteo_data, sfincs_meteo.f90:35-98, 330-412).
struct SpwGrid {
  int nt, nrows, ncols, precip;  // precip: the fourth quantity is used as rain
  float radius, drad, dphi, merge_frac;
  const float* times;  // [nt] seconds after tref
  const float* xe;     // [nt] eye position
  const float* ye;
  const float* wu;     // [nt][nrows][ncols] wind components (m/s), rows outward, columns clockwise from north
  const float* wv;
  const float* pabs;   // absolute pressure (Pa)
  const float* prcp;   // rain (mm/h), when precip
};

struct ScnDev {
  // ---- grid
  int nmax, mmax, ld, subgrid;
  int64_t nalloc;
  float dx, dy, dxinv, dyinv, dx2inv, dy2inv, area;
  // ---- physics switches and parameters (sfincs_input.f90 defaults)
  float g, huthresh, huvmin, alfa, uvlim, advlim, slopelim, wiggle_threshold, wiggle_factor, theta;
  float nuvisc, nuviscfac, fcorio, dtmax, dtmin, rhoa, rhow, btfilter, btrelax, zini, tspinup, t0, t1;
  int advection, adv_scheme, viscosity, coriolis, friction2d, thetasmooth, wiggle, wind, precip, use_qext;
  int store_zsmax, infiltration, nlev, nref;
  // ---- state
  float* zs;
  float* zsmax;
  double* zvol;
  float* zs0;
  float* zsderv;
  uint8_t* kf[2];      // wet history of the u / v face owned by each cell
  uint8_t* vneg;       // subgrid: z_volume < 0 (written by continuity)
  float* qu[2];
  float* qv[2];
  float* uu[2];
  float* vv[2];
  const uint16_t* flags;
  // ---- regular bathymetry
  const float* zb;
  const float* zbmx_u;   // zbuvmx of the u face
  const float* zbmx_v;
  const float* gn2_u;
  const float* gn2_v;
  // ---- subgrid tables
  const float2* sgz_u;   // (zmin, zmax) of the u face
  const float2* sgz_v;
  const float4* sgw_u;   // (havg_zmax, nrep_zmax, navg_w, fnfit)
  const float4* sgw_v;
  const UvRec* rec_u;    // [level k = 0..nlev-2][cell offset]
  const UvRec* rec_v;
  const float* zz_min;
  const float* zz_max;
  const float* zz_volmax;
  const float2* zlev;    // [level][cell]: (dep_k, dep_k+1 - dep_k)
  // Per-face record cache (regular subgrid grids, TMA kernels): the table
  // values the face used last step, in two arrays so that a warp reads whole
  // lines with one 16-byte and one 8-byte load per face: rc4 = (havg, dhavg,
  // nrep, dnrep) of level k or the full-branch coefficients sgw, rc2 = (pwet,
  // dpwet); rl: what they hold, 0 = nothing, k + 1 = level k, kRecFull = the
  // full branch.  Both depend on (face, level) only, so an entry never goes
  // stale.
  float4* rc4_u;
  float4* rc4_v;
  float2* rc2_u;
  float2* rc2_v;
  uint8_t* rl_u;
  uint8_t* rl_v;
  // The same for the volume-to-level inversion: zc holds the z_level pair of
  // interval zl - 1 (zl = 0: nothing cached).
  float2* zc;
  uint8_t* zl;
  // ---- per-cell forcing
  const float* qext;
  const float* qinf;     // infiltration field (m/s), con/c2d
  // ---- boundary forcing
  int nbnd, ntbnd, nkcuv2, nneu, ngbnd;
  const float* t_bnd;    // [ntbnd]
  const float* zs_bnd;   // [ntbnd][nbnd]
  float* zst_bnd;        // [nbnd] levels at the boundary points for the current step
  int ntide;             // astronomic constituents per boundary point (0: none; the first is A0)
  const double* tide_w;  // [ntide] frequency (rad/s)
  const double* tide_amp;  // [nbnd][ntide] amplitude times nodal factor
  const double* tide_pha;  // [nbnd][ntide] phase less V0+u (rad)
  const BndFace* bfaces; // [nkcuv2]
  float* uvmean;         // [nkcuv2]
  const int2* neu;       // [nneu] Neumann (kcs 6) cell and its interior cell (dense offsets)
  // ---- time series (uniform meteo, point sources)
  int ntprcp, ntwnd, nsrc, ntsrc;
  const float* tprcp;
  const float* vprcp;
  const float* twnd;
  const float* wmag;
  const float* wdir;
  const float* cdval;    // [1000]
  const float* tsrc;
  const float* qsrc;     // [ntsrc][nsrc]
  float* qtsrc;          // [nsrc]
  const int* src_cell;   // [nsrc]
  int nstruc;            // weir faces
  const StrucFace* struc;  // [nstruc]
  int ndrn;              // drainage structures; qtsrc and src_cell hold nsrc + 2 ndrn entries (intake, outfall per structure)
  const DrnDev* drn;     // [ndrn]
  int* drn_status;       // [ndrn] gates: 0 closed, 1 open, 2 closing, 3 opening
  float* drn_frac;       // [ndrn] gates: fraction open
  float structure_relax; // seconds
  float pi;
  // store variables (compute_store_variables, sfincs_continuity.f90:626-720, and
  // t_zsmax, :239-255): maximum cell velocity and flux, wet duration, time of
  // the maximum level; dense per-cell arrays, null when off
  int store_vmax, store_qmax, store_twet, store_tzsmax;
  float twet_threshold;
  float* vmax;
  float* qmax;
  float* twet;
  float* tzsmax;
  // Infiltration with state (update_infiltration_map, sfincs_infiltration.f90:
  // 678-1033): inftype 2 curve number (cna), 3 curve number with recovery
  // (cnb), 4 Green-Ampt (gai), 5 Horton (hor); con / c2d (inftype 1) use qinf.
  // Per-cell parameters and state, dense like the other cell arrays:
  //   cna: par 0 S (m)
  //   cnb: par 0 Smax, 1 recovery rate kr; state 0 Se, 1 P1, 2 F1, 3 S1, 4 T1; rain flag
  //   gai: par 0 ks (m/s), 1 sigma_max, 2 Lu (m), 3 kr, 4 suction head (m); state 0 sigma, 1 F, 2 T1, 3 qinfmap
  //   hor: par 0 fc, 1 f0 (mm/h), 2 kd (1/h); state 0 T1
  int inftype, store_cumprcp;
  float sfacinf, horton_kr_kd;
  int64_t inf_last;      // storage index of the model's last cell (gai reads its head and sigma)
  const float* inf_par[5];
  float* inf_st[5];
  uint8_t* inf_rain;
  // geographic grids (crsgeo, sfincs_domain.f90:1403-1473; null on projected
  // grids): per cell its width dxm (m), 1/dxm (the inverse spacing of both of
  // its faces across x), its area (m2) and its Coriolis parameter
  int geo;
  float geo_dyrm;        // 111111.1 dy (m): the length of the u faces
  const float* geo_dxm;
  const float* geo_dxminv;
  const float* geo_area;
  const float* geo_fcor;
  float* qinfmap;        // infiltration rate of the step (m/s) per cell, when an output needs it (else null)
  float* cumprcp;        // cumulative rain and infiltration (m), when stored or needed (cna, cnb)
  float* cuminf;
  // gridded meteo (sfincs_meteo.f90:802-1442): the raw grids (0 wind, 1
  // pressure, 2 rain), the cell centres they are interpolated to (compact
  // order, cmp: compact cell -> storage offset, null when they coincide), the
  // two fields of the current update window per cell, and the switches
  int meteo3d, patmos, wind_field, prcp_field, spinup_meteo, ampr_block;
  int nmeteo;            // cells the fields cover (compact count)
  float dtwnd, gapres, pavbnd, cosrot, sinrot;
  MeteoGrid mg[3];
  SpwGrid spw;           // nt == 0: none
  const float* xz;
  const float* yz;
  const int32_t* cmp;
  float* tauwu0;
  float* tauwu1;
  float* tauwv0;
  float* tauwv1;
  float* patm0;
  float* patm1;
  float* prcp0;
  float* prcp1;
  int wait_limit;        // try_wait rounds of a staged kernel's bounded wait for its tile data (2^22)
  int h73table;          // hu**(7/3) from the lookup table (sfincs_momentum.f90:663-675)
  const float* x73;      // [10][1000] the table x73(j, k) at (k - 1) * 1000 + j - 1 (sfincs_data.f90:858-881)
  StepState* st;
  // ---- quadtree (quadtree != 0; the regular-grid fields above that index
  // cells or faces then hold compact arrays: zs.. over npc cells, qu/qv and
  // uu/vv both point at the one q / uv array, kf[0] = kfuv, sgz_u/v, sgw_u/v
  // and rec_u/v at the face tables with nalloc = npuv as the level stride)
  int quadtree, npc, npuv, ncuv;
  const FaceQ* qface;   // [npuv]
  const int4* qcell;    // [npc] q index of the md, mu, nd, nu uv point of each cell
  const int2* qcuv;     // [ncuv] q indices of the two fine faces of combined point npuv + i
  const uint8_t* qlev;  // [npc] refinement level - 1
  const float* zbmx;    // [npuv] regular bed: zbuvmx
  const float* gn2;     // [npuv] regular bed: g n^2
  float lv_dxrinv[kMaxQtLevels], lv_dyrinv[kMaxQtLevels], lv_dxr2inv[kMaxQtLevels], lv_dyr2inv[kMaxQtLevels];
  float lv_dxrinvc[kMaxQtLevels], lv_dyrinvc[kMaxQtLevels], lv_dxrm[kMaxQtLevels], lv_dyrm[kMaxQtLevels];
  float lv_area[kMaxQtLevels], lv_nuvisc[kMaxQtLevels], lv_nuvisc_t[kMaxQtLevels];
};

struct Tile {  // one CTA of the cell kernels
  int scn, n0, m0, pad;
};

// TMA tensor maps of one scenario (2-D views of the dense arrays, boxes sized
// for 32 x 8 cell tiles plus the halo each kernel needs).  The maps live in
// device memory, 64-byte aligned, one MapSet per scenario.
enum MapId : int {
  // momentum
  MM_ZS, MM_QU0, MM_QU1, MM_QV0, MM_QV1, MM_UU0, MM_UU1, MM_VV0, MM_VV1, MM_FLAGS, MM_KFU, MM_KFV,
  MM_VNEG, MM_ZSD, MM_SGZU, MM_SGZV, MM_ZB, MM_ZBMXU, MM_ZBMXV, MM_GN2U, MM_GN2V, MM_RLU, MM_RLV,
  // continuity
  MC_QU0, MC_QU1, MC_QV0, MC_QV1, MC_ZS, MC_ZSMAX, MC_ZVOL, MC_ZS0, MC_VOLMAX, MC_VNEG, MC_FLAGS, MC_QEXT,
  MC_QINF, MC_ZB, MC_ZL, MC_ZZMIN, MC_ZZMAX, MC_ZC,
  NUM_MAPS
};
struct alignas(64) MapSet {
  unsigned char m[NUM_MAPS][128];  // CUtensorMap objects (opaque, 128 bytes each)
};

#ifdef __CUDACC__
// The step scalars a cell or face update reads, copied into registers once per
// scenario instead of being re-read from the step state for every cell.
struct StepVals {
  float dt, ptmp, twu, twv;
  int parity;
};
__device__ __forceinline__ StepVals step_vals(const StepState& st) {
  return StepVals{st.dt, st.ptmp, st.twu, st.twv, st.parity};
}

// 1-based table interval int(x) + 1 of a subgrid lookup (sfincs_momentum.f90:
// 372-378, sfincs_continuity.f90:566), clamped to [1, nlev - 1].  For every
// finite x that the callers' guards let through the interval is already in
// that range, so the clamp changes no result.  It matters for non-finite state
// after a model has gone unstable: the guards pass NaN to the interval branch,
// and an f64 NaN converts to INT_MIN (an f32 NaN to 0), which would otherwise
// index far outside the table.
// Store variables of one kcs == 1 cell after its continuity update
// (compute_store_variables, sfincs_continuity.f90:626-720): the cell-centre
// velocity and flux magnitudes from the means of the cell's two u and two v
// faces (this step's values), and the wet duration.  uv_* are read by the
// caller only when vmax is stored; base is zb or the subgrid z_zmin.
__device__ __forceinline__ void store_cell_variables(const ScnDev& S, int64_t c, float q_md, float q_mu, float q_nd,
                                                     float q_nu, float uv_md, float uv_mu, float uv_nd, float uv_nu,
                                                     float zsn, float base, float dt) {
  if (S.store_vmax) {
    const float quz = (uv_md + uv_mu) / 2.0f, qvz = (uv_nd + uv_nu) / 2.0f;
    const float uvz = sqrtf(quz * quz + qvz * qvz);
    S.vmax[c] = fmaxf(S.vmax[c], uvz);
  }
  if (S.store_qmax) {
    const float quz = (q_md + q_mu) / 2.0f, qvz = (q_nd + q_nu) / 2.0f;
    const float qz = sqrtf(quz * quz + qvz * qvz);
    S.qmax[c] = fmaxf(S.qmax[c], qz);
  }
  if (S.store_twet && (double)zsn - (double)base > (double)S.twet_threshold) S.twet[c] = S.twet[c] + dt;
}
// Time of the maximum level (:239-255): set where the new level exceeds the
// stored maximum and the cell is wet by more than huthresh; zm is the maximum
// before this step's update.
__device__ __forceinline__ void store_tzsmax(const ScnDev& S, int64_t c, float zsn, float zm, float base) {
  if (zsn > zm && (double)zsn - (double)base > (double)S.huthresh) S.tzsmax[c] = (float)S.st->t;
}

// Time weights of the gridded meteo fields at model time t
// (update_meteo_forcing, sfincs_meteo.f90:1272-1274, 1349-1352): the window
// weight and, while the meteo spins up, the spin-up factor.
struct MeteoW {
  float twf, smf;
  bool spin;
};
__device__ __forceinline__ MeteoW meteo_weights(const ScnDev& S, double t, float mt0, float mt1) {
  MeteoW w;
  w.twf = (float)((t - (double)mt0) / (double)(mt1 - mt0));
  w.spin = S.spinup_meteo && t < (double)(S.tspinup - 1.0e-3f);
  w.smf = w.spin ? (float)((t - (double)S.t0) / (double)(S.tspinup - S.t0)) : 1.0f;
  return w;
}
// Pressure of storage cell c this step (:1302-1304, 1364-1366).
__device__ __forceinline__ float cell_patm(const ScnDev& S, int64_t c, const MeteoW& w) {
  float p = S.patm0[c] * (1.0f - w.twf) + S.patm1[c] * w.twf;
  if (w.spin) p = p * w.smf + S.gapres * (1.0f - w.smf);
  return p;
}
// Wind stress of storage cell c in direction dir this step (:1282-1288, 1357-1360).
__device__ __forceinline__ float cell_tau(const ScnDev& S, int64_t c, int dir, const MeteoW& w) {
  const float* a = dir == 0 ? S.tauwu0 : S.tauwv0;
  const float* b = dir == 0 ? S.tauwu1 : S.tauwv1;
  float tw = a[c] * (1.0f - w.twf) + b[c] * w.twf;
  if (w.spin) tw = tw * w.smf;
  return tw;
}
// Rain of storage cell c this step (:1306-1330, 1368-1394): prcp, and the net
// rain before infiltration; negative rain is dropped on a dry cell.
__device__ __forceinline__ float cell_rain(const ScnDev& S, int64_t c, const MeteoW& w, bool dry, float& net) {
  float pr = S.prcp0[c] * (1.0f - w.twf) + S.prcp1[c] * w.twf;
  if (pr < 0.0f && dry) pr = 0.0f;
  net = pr;
  if (w.spin) {
    net = net * w.smf;
    if (net < 0.0f && dry) net = 0.0f;
  }
  return pr;
}

// The step's infiltration rate of an active cell (qinfmap,
// sfincs_infiltration.f90:632-1033), kept when an output needs it: the rate
// of the model with state, else the constant / c2d rate on a wet cell.
__device__ __forceinline__ void store_qinfmap(const ScnDev& S, int64_t c, bool inf_cell, float qinf_cell, bool wet) {
  S.qinfmap[c] = inf_cell ? qinf_cell : ((S.infiltration && wet) ? S.qinf[c] : 0.0f);
}

// Cosine in FP64 from IEEE operations only, so that the oracle reproduces it
// bit for bit: n = rint(x 2/pi); r = x - n pi/2 with pi/2 split in three
// doubles (Cody and Waite, each product fused with its subtraction), so r is
// within an ulp for |n| far beyond any tidal argument; then the Taylor series
// of sin (to degree 17) or cos (to degree 18) of r in [-pi/4, pi/4], in Horner
// form, by the quadrant n mod 4.  Truncation stays below 1e-19.
__device__ __forceinline__ double cos_ieee(double x) {
  const double n = rint(__dmul_rn(x, 0.6366197723675814));
  double r = __fma_rn(-n, 1.5707963267948966, x);
  r = __fma_rn(-n, 6.123233995736766e-17, r);
  r = __fma_rn(-n, -1.4973849048591698e-33, r);
  const double r2 = __dmul_rn(r, r);
  const int q = (int)((long long)n & 3);
  if (q & 1) {  // +-sin(r)
    double p = 2.8114572543455206e-15;
    p = __fma_rn(p, r2, -7.647163731819816e-13);
    p = __fma_rn(p, r2, 1.6059043836821613e-10);
    p = __fma_rn(p, r2, -2.505210838544172e-08);
    p = __fma_rn(p, r2, 2.7557319223985893e-06);
    p = __fma_rn(p, r2, -0.0001984126984126984);
    p = __fma_rn(p, r2, 0.008333333333333333);
    p = __fma_rn(p, r2, -0.16666666666666666);
    const double sn = __fma_rn(__dmul_rn(r, r2), p, r);
    return q == 1 ? -sn : sn;
  }
  double p = -1.5619206968586225e-16;
  p = __fma_rn(p, r2, 4.779477332387385e-14);
  p = __fma_rn(p, r2, -1.1470745597729725e-11);
  p = __fma_rn(p, r2, 2.08767569878681e-09);
  p = __fma_rn(p, r2, -2.755731922398589e-07);
  p = __fma_rn(p, r2, 2.48015873015873e-05);
  p = __fma_rn(p, r2, -0.001388888888888889);
  p = __fma_rn(p, r2, 0.041666666666666664);
  p = __fma_rn(p, r2, -0.5);
  const double cs = __fma_rn(r2, p, 1.0);
  return q == 0 ? cs : -cs;
}

// Level of boundary point ib with its astronomic constituents added one by one
// in FP64, each sum rounded to the point's real*4 level (sfincs_boundaries.f90:736-744).
__device__ __forceinline__ float tide_level(const ScnDev& S, int ib, double t, float z) {
  const double* a = S.tide_amp + (size_t)ib * S.ntide;
  const double* ph = S.tide_pha + (size_t)ib * S.ntide;
  for (int c = 0; c < S.ntide; c++) {
    const double arg = __dsub_rn(__dmul_rn(S.tide_w[c], t), ph[c]);
    z = (float)__dadd_rn((double)z, __dmul_rn(a[c], cos_ieee(arg)));
  }
  return z;
}

// Four-quadrant arctangent from IEEE operations only, so that the oracle
// reproduces it bit for bit: a = min(|x|,|y|) / max(|x|,|y|) in [0, 1]; above
// tan(pi/12) the addition formula atan(a) = pi/6 + atan((sqrt3 a - 1) / (sqrt3 + a))
// brings the argument into [-tan(pi/12), tan(pi/12)], where the Taylor series
// of atan to degree 15 (Horner form) leaves a truncation error below 1e-11;
// the octant and the quadrant follow from the signs and from |y| > |x|.
// atan2(0, 0) is 0.
__device__ __forceinline__ float atan2_ieee(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  if (mx == 0.0f) return 0.0f;
  const float a = mn / mx;
  float t = a, off = 0.0f;
  if (a > 0.267949194f) {
    t = (1.73205081f * a - 1.0f) / (1.73205081f + a);
    off = 0.523598776f;
  }
  const float t2 = t * t;
  float p = -1.0f / 15.0f;
  p = fmaf(p, t2, 1.0f / 13.0f);
  p = fmaf(p, t2, -1.0f / 11.0f);
  p = fmaf(p, t2, 1.0f / 9.0f);
  p = fmaf(p, t2, -1.0f / 7.0f);
  p = fmaf(p, t2, 1.0f / 5.0f);
  p = fmaf(p, t2, -1.0f / 3.0f);
  float r = off + fmaf(t * t2, p, t);
  if (ay > ax) r = 1.57079633f - r;
  if (x < 0.0f) r = 3.14159265f - r;
  return y < 0.0f ? -r : r;
}

// Exponential from IEEE operations only, so that the oracle reproduces it bit
// for bit: n = rint(x log2 e), r = x - n ln2 with ln2 split in two parts
// (Cody and Waite), e^r by its Taylor polynomial to degree 7 in Horner form,
// times 2^n applied as two exact powers of two.  Within 0.94 ulp of e^x for
// -87 <= x <= 88.7.
__device__ __forceinline__ float exp_ieee(float x) {
  if (x != x) return x;
  if (x > 88.8f) return __int_as_float(0x7f800000);
  if (x < -104.0f) return 0.0f;
  const float n = rintf(x * 1.44269502f);
  float r = fmaf(-n, 0.693145752f, x);
  r = fmaf(-n, 1.42860677e-06f, r);
  float p = 1.98412701e-04f;
  p = fmaf(p, r, 1.38888892e-03f);
  p = fmaf(p, r, 8.33333377e-03f);
  p = fmaf(p, r, 4.16666679e-02f);
  p = fmaf(p, r, 1.66666672e-01f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  const int ni = (int)n, n1 = ni / 2, n2 = ni - n1;
  return (p * __int_as_float((n1 + 127) << 23)) * __int_as_float((n2 + 127) << 23);
}

// Infiltration of one active cell in this step (update_infiltration_map,
// sfincs_infiltration.f90:609-1039, with the cumulative rain of
// update_precipitation_from_timeseries, sfincs_meteo.f90:1545-1547); returns
// qinfmap (m/s) and updates the cell's state.  dry: no water in the cell
// (con / c2d), hh: the local depth estimate (Horton), ga_hs: the Green-Ampt
// product GA_head(np) * GA_sigma(np) that the reference uses for every cell.
__device__ __forceinline__ float cell_infiltration(const ScnDev& S, int64_t c, float prcp, float dt, bool dry,
                                                   float hh, float ga_hs) {
  if (S.store_cumprcp) S.cumprcp[c] = S.cumprcp[c] + prcp * dt;
  float q = 0.0f;
  if (S.inftype == 1) {  // con / c2d (:632-676)
    q = dry ? 0.0f : S.qinf[c];
  } else if (S.inftype == 2) {  // cna (:678-723)
    const float cp = S.cumprcp[c], Sv = S.inf_par[0][c];
    if (cp > S.sfacinf * Sv) {
      const float a = cp - S.sfacinf * Sv;
      const float Qq = a * a / (cp + (1.0f - S.sfacinf) * Sv);
      q = ((cp - Qq) - S.cuminf[c]) / dt;
    } else {
      q = prcp;
    }
  } else if (S.inftype == 3) {  // cnb (:724-829)
    float se = S.inf_st[0][c], t1 = S.inf_st[4][c];
    if (prcp > 0.0f) {
      float p1 = S.inf_st[1][c], f1 = S.inf_st[2][c], s1 = S.inf_st[3][c];
      if (S.inf_rain[c] != 1) {  // a new rain event
        p1 = 0.0f;
        f1 = 0.0f;
        s1 = se;
        S.inf_rain[c] = 1;
        S.inf_st[3][c] = s1;
      }
      p1 = p1 + prcp * dt;
      if (p1 > S.sfacinf * s1) {
        const float a = p1 - S.sfacinf * s1;
        const float Qq = a * a / (p1 + (1.0f - S.sfacinf) * s1);
        const float I = p1 - Qq;
        q = (I - f1) / dt;
        f1 = I;
      } else {
        f1 = p1;
        q = prcp;
      }
      se = fmaxf(se - q * dt, 0.0f);
      q = fmaxf(q, 0.0f);
      S.inf_st[1][c] = p1;
      S.inf_st[2][c] = f1;
    } else {
      if (S.inf_rain[c] == 1) {  // the event ended
        S.inf_rain[c] = 0;
        t1 = 0.0f;
      }
      t1 = t1 + dt / 3600.0f;
      const float kr = S.inf_par[1][c], smax = S.inf_par[0][c];
      if (t1 > 0.06f / kr) {  // recovery (SWMM equation 4-37)
        se = se + kr * smax * dt / 3600.0f;
        se = fminf(se, smax);
      }
    }
    S.inf_st[0][c] = se;
    S.inf_st[4][c] = t1;
  } else if (S.inftype == 4) {  // gai (:830-912); the rate is kept while it does not rain
    float sig = S.inf_st[0][c], F = S.inf_st[1][c], t1 = S.inf_st[2][c];
    const float kr = S.inf_par[3][c], smax = S.inf_par[1][c], Lu = S.inf_par[2][c];
    if (prcp > 0.0f) {
      const float ks = S.inf_par[0][c];
      if (prcp < ks) {
        q = prcp;
      } else {
        q = ks * (1.0f + ga_hs / F);
        q = fmaxf(fminf(q, prcp), 0.0f);
      }
      sig = fmaxf(sig - q * dt / Lu, 0.0f);
      F = F + q * dt;
      t1 = 0.0f;
      S.inf_st[3][c] = q;
    } else {
      q = S.inf_st[3][c];
      t1 = t1 + dt / 3600.0f;
      if (t1 > 0.06f / kr) {
        sig = sig + kr * smax * dt / 3600.0f;
        sig = fminf(sig, smax);
        F = fmaxf(F - kr * smax * dt / 3600.0f * Lu, 0.0f);
      }
    }
    S.inf_st[0][c] = sig;
    S.inf_st[1][c] = F;
    S.inf_st[2][c] = t1;
  } else if (S.inftype == 5) {  // hor (:914-1033)
    float t1 = S.inf_st[0][c];
    if (hh > 0.0f || prcp > 0.0f) {
      t1 = t1 > 0.0f ? 0.0f : t1 - dt;
      const float fc = S.inf_par[0][c];
      float I = exp_ieee(S.inf_par[2][c] * t1 / 3600.0f);
      if (I < 0.01f) {
        t1 = t1 + dt;
        q = fc / 3600.0f / 1000.0f;
      } else {
        q = (fc + (S.inf_par[1][c] - fc) * I) / 3600.0f / 1000.0f;
      }
      const float Qq = hh > 0.0f ? prcp * dt + hh : prcp * dt;
      I = q * dt;
      if (I > Qq) q = q * Qq / I;
    } else {
      t1 = t1 + dt / S.horton_kr_kd;
    }
    S.inf_st[0][c] = t1;
  }
  if (S.store_cumprcp && S.inftype >= 1) S.cuminf[c] = S.cuminf[c] + q * dt;
  return q;
}

__device__ __forceinline__ int lev_index(float x, int nlev) { return min(max((int)x + 1, 1), nlev - 1); }
__device__ __forceinline__ int lev_index(double x, int nlev) { return min(max((int)x + 1, 1), nlev - 1); }
#endif

}  // namespace sfg
