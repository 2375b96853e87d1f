// TMA-staged momentum and continuity kernels (sm_100a).
//
// Same arithmetic as kernels.cu (sfincs_momentum.f90:157-752,
// sfincs_continuity.f90:46-624), different memory pipeline: persistent CTAs of
// 256 threads walk the tile table with a stride of gridDim.x; for every 32 x 8
// cell tile one elected thread issues one 2-D cp.async.bulk.tensor load per
// state array (the tile plus the one-cell halo the stencil reads) into a shared
// memory stage, completing on an mbarrier.  Two stages: the next tile streams in
// while the current one is computed.  Only the data-dependent subgrid table
// records are still read with per-thread loads.
//
// All TMA coordinates keep the innermost coordinate a multiple of 16 bytes
// (tile origins are 128-byte aligned, halos are rounded down to 4 floats / 8
// half-words / 16 bytes), loads only (no TMA stores, no cluster multicast).
// Every mbarrier wait is bounded: on timeout the CTA records a fault in the
// scenario's step state, skips the tile and later drains its copies (bounded).
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "face_math.h"
#include "pdl.h"
#include "sfg_device.h"

namespace sfg {

// --------------------------------------------------------------------------
// PTX helpers
// --------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: `limit` try_wait rounds (each already suspends for a while)
// before giving up; the scenario's wait_limit is 2^22 unless a test lowers it.
constexpr int kDrainRounds = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// A wait that gave up leaves its stage's copies in flight.  The CTA then
// issues no further loads (every tile it still visits is skipped), and
// before it exits thread 0 waits (bounded) for the last phase of every
// stage: each issued phase has been waited for in the loop, so when those
// waits succeeded each of these returns at the first try_wait (a stage never
// loaded has completed its phase of parity 1).
__device__ __noinline__ void drain_stages(uint64_t* bar, int nst, uint32_t phase) {
  for (int k = 0; k < nst; k++) (void)mbar_wait_bounded(&bar[k], ((phase >> k) & 1u) ^ 1u, kDrainRounds);
}
__device__ __forceinline__ void tma_load_2d(void* dst, const void* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ float warp_max_t(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Running CFL terms of a thread's faces: the largest g*hu and |uv| of its u
// faces and of its v faces (see face_flux_geo: max over faces commutes with the
// monotone sqrt and the multiplication by the spacing).  A flush folds a warp's
// terms into the scenario's min_dt: one division and one atomicMin per warp
// (positive floats order like their bits).
struct CflTerms {
  float ghu_u = 0.0f, uv_u = 0.0f, ghu_v = 0.0f, uv_v = 0.0f;
};
__device__ __forceinline__ void flush_cfl(StepState* st, const CflTerms& t, float dxinv, float dyinv, int lane) {
  const float den_u = fmaxf(sqrtf(warp_max_t(t.ghu_u)), warp_max_t(t.uv_u)) * dxinv;
  const float den_v = fmaxf(sqrtf(warp_max_t(t.ghu_v)), warp_max_t(t.uv_v)) * dyinv;
  const float den = fmaxf(den_u, den_v);
  if (lane == 0 && st && den > 0.0f) atomicMin(&st->min_dt_bits, __float_as_uint(1.0f / den));
}

// --------------------------------------------------------------------------
// Shared-memory stage layouts (byte offsets; every box starts 128-byte aligned)
// --------------------------------------------------------------------------
namespace mom {
// box widths / heights and the tile origin inside each box
// zs/zsderv/zb: 36 x 9 (n0..n0+35, m0..m0+8); qu: 36 x 10 (m0-1..m0+8);
// qv: 40 x 9 (n0-4..n0+35); uu, vv: 40 x 10 (n0-4.., m0-1..)
constexpr int W_ZS = 36, W_QU = 36, W_QV = 40, W_UV = 40;
constexpr int O_ZS = 0, O_QU = 1408, O_QV = 2944, O_UU = 4480, O_VV = 6144, O_FLAGS = 7808, O_KFU = 8320,
              O_KFV = 8576;
constexpr int O_VNEG = 8832, O_ZSD = 9344, O_SGZU = 10752, O_SGZV = 12800;       // subgrid
// subgrid record-cache codes: one byte per face (the 16 + 8-byte entries are read per thread)
constexpr int O_RLU = 14848, O_RLV = 15104;
constexpr int O_ZB = 8832, O_ZBMXU = 10240, O_ZBMXV = 11264, O_GN2U = 12288, O_GN2V = 13312;  // regular
constexpr int STAGE = 14848, STAGE_SG = 15360;
template <bool SG>
__host__ __device__ constexpr int stage_bytes() { return SG ? STAGE_SG : STAGE; }
constexpr uint32_t B_COMMON = 36 * 9 * 4 + 36 * 10 * 4 + 40 * 9 * 4 + 2 * 40 * 10 * 4 + 32 * 8 * 2 + 2 * 32 * 8;
}  // namespace mom

namespace con {
constexpr int O_QU = 0, O_QV = 1152, O_ZS = 2304, O_ZSMAX = 3328, O_FLAGS = 4352, O_ZVOL = 4864, O_VOLMAX = 6912,
              O_VNEG = 7936, O_ZS0 = 8192, O_QEXT = 9216, O_QINF = 10240, O_ZB = 11264, O_ZL = 12288,
              O_ZZMIN = 12544, O_ZZMAX = 13568, O_ZC = 14592;  // subgrid: z_zmin, z_zmax, z_level cache
constexpr int STAGE = 16640;
}  // namespace con

__device__ __forceinline__ const void* map_of(const MapSet* maps, int scn, int id) { return maps[scn].m[id]; }

// Where a tile's scenario parameters come from.  ONE: the launch advances a
// single model whose ScnDev is passed by value as a __grid_constant__ kernel
// parameter, so every field is a constant-bank operand (no load instruction,
// no address arithmetic, no aliasing with the stores of the step).  Otherwise
// the device table of an ensemble, indexed by the tile's scenario.
template <bool ONE>
__device__ __forceinline__ const ScnDev& scn_of(const ScnDev* __restrict__ scns, const ScnDev& one, int i) {
  if (ONE) return one;
  return scns[i];
}

// --------------------------------------------------------------------------
// Momentum
// --------------------------------------------------------------------------
template <bool SG>
__device__ __forceinline__ bool issue_momentum(const ScnDev& S, const MapSet* maps, const Tile& tl,
                                               unsigned char* st, uint64_t* bar) {
  const StepState& ss = *S.st;
  if (!ss.run) return false;
  const int p = ss.parity;
  const int x = kGhostPad + tl.n0;  // multiple of 32
  const int y = tl.m0;
  uint32_t bytes = mom::B_COMMON;
  if (SG) bytes += 48 * 9 + 2 * 64 * 8 * 4 + 2 * 32 * 8 + (S.wiggle ? 36 * 9 * 4 : 0);
  else bytes += 36 * 9 * 4 + 4 * 32 * 8 * 4;
  mbar_expect_tx(bar, bytes);
  tma_load_2d(st + mom::O_ZS, map_of(maps, tl.scn, MM_ZS), x, y, bar);
  tma_load_2d(st + mom::O_QU, map_of(maps, tl.scn, MM_QU0 + p), x, y - 1, bar);
  tma_load_2d(st + mom::O_QV, map_of(maps, tl.scn, MM_QV0 + p), x - 4, y, bar);
  tma_load_2d(st + mom::O_UU, map_of(maps, tl.scn, MM_UU0 + p), x - 4, y - 1, bar);
  tma_load_2d(st + mom::O_VV, map_of(maps, tl.scn, MM_VV0 + p), x - 4, y - 1, bar);
  tma_load_2d(st + mom::O_FLAGS, map_of(maps, tl.scn, MM_FLAGS), x, y, bar);
  tma_load_2d(st + mom::O_KFU, map_of(maps, tl.scn, MM_KFU), x, y, bar);
  tma_load_2d(st + mom::O_KFV, map_of(maps, tl.scn, MM_KFV), x, y, bar);
  if (SG) {
    tma_load_2d(st + mom::O_VNEG, map_of(maps, tl.scn, MM_VNEG), x, y, bar);
    if (S.wiggle) tma_load_2d(st + mom::O_ZSD, map_of(maps, tl.scn, MM_ZSD), x, y, bar);
    tma_load_2d(st + mom::O_SGZU, map_of(maps, tl.scn, MM_SGZU), 2 * x, y, bar);
    tma_load_2d(st + mom::O_SGZV, map_of(maps, tl.scn, MM_SGZV), 2 * x, y, bar);
    tma_load_2d(st + mom::O_RLU, map_of(maps, tl.scn, MM_RLU), x, y, bar);
    tma_load_2d(st + mom::O_RLV, map_of(maps, tl.scn, MM_RLV), x, y, bar);
  } else {
    tma_load_2d(st + mom::O_ZB, map_of(maps, tl.scn, MM_ZB), x, y, bar);
    tma_load_2d(st + mom::O_ZBMXU, map_of(maps, tl.scn, MM_ZBMXU), x, y, bar);
    tma_load_2d(st + mom::O_ZBMXV, map_of(maps, tl.scn, MM_ZBMXV), x, y, bar);
    tma_load_2d(st + mom::O_GN2U, map_of(maps, tl.scn, MM_GN2U), x, y, bar);
    tma_load_2d(st + mom::O_GN2V, map_of(maps, tl.scn, MM_GN2V), x, y, bar);
  }
  return true;
}

// Regular-grid face of direction DIR: spacing and switches from the scenario
// and the cell's flag bits.
template <bool SG, int DIR, bool MET>
__device__ __forceinline__ float face_flux(const ScnDev& S, const StepVals& st, uint16_t f, uint8_t kf, float zs_nm,
                                           float zs_nmu, float hu, float gnavg2, float phi, const FaceV& a,
                                           bool dry_nm, bool dry_nmu, float zd_nm, float zd_nmu, int64_t c,
                                           float& q_out, float& uv_out) {
  constexpr uint16_t ADV = DIR == 0 ? F_UADV : F_VADV;
  constexpr uint16_t TH = DIR == 0 ? F_UTH : F_VTH;
  FaceGeo geo;
  geo.dxuvinv = DIR == 0 ? S.dxinv : S.dyinv;
  geo.dyuvinv = DIR == 0 ? S.dyinv : S.dxinv;
  geo.dxuv2inv = DIR == 0 ? S.dx2inv : S.dy2inv;
  geo.dyuv2inv = DIR == 0 ? S.dy2inv : S.dx2inv;
  geo.nuvisc = S.nuvisc;
  geo.fcorio = S.fcorio;
  // MET: a gridded wind or pressure field is present (a separate kernel
  // instance, so that the plain path keeps its register allocation)
  float tauw = DIR == 0 ? st.twu : st.twv, dpatm = 0.0f;
  if (MET) face_meteo(S, st, DIR, c, DIR == 0 ? c + S.ld : c + 1, tauw, dpatm);
  return face_flux_geo<SG>(S, st, DIR, (f & ADV) != 0, (f & TH) != 0, geo, kf, zs_nm, zs_nmu, hu, gnavg2, phi, a,
                           dry_nm, dry_nmu, zd_nm, zd_nmu, tauw, dpatm, q_out, uv_out);
}

// Subgrid depth / roughness / wet fraction at the face level zsu (sfincs_momentum.f90:345-380).
// full (zsu above the table): v = (havg_zmax, nrep_zmax, navg_w, fnfit) of the face;
// otherwise v = (havg, dhavg, nrep, dnrep) and v2 = (pwet, dpwet) of level interval iuv.
struct SgLook {
  float4 v;
  float2 v2;
  float facint;
  bool full;
};

// Thread 0 reads each tile's header when it issues the tile's loads and passes
// it on through shared memory; the step scalars are read once per scenario.
// NST stages: the loads of a tile are issued NST - 1 tiles before its update
// (one CTA barrier per tile orders the reuse of a stage).
template <bool SG, int MINB, bool ONE, int NST, bool MET>
__global__ void __launch_bounds__(256, MINB) k_momentum_tma(const ScnDev* __restrict__ scns,
                                                            const MapSet* __restrict__ maps,
                                                            const Tile* __restrict__ tiles, int ntiles,
                                                            const __grid_constant__ ScnDev one) {
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[NST];
  __shared__ int s_issued[NST];
  __shared__ Tile s_tile[NST];
  __shared__ int s_stop;  // a wait of this CTA ran out
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + 32 * ty;
  const int G = gridDim.x;
  int tile = blockIdx.x;
  // thread 0: load tile t into stage k
  auto issue = [&](int t, int k) {
    if (t < ntiles) {
      const Tile tn = tiles[t];
      s_tile[k] = tn;
      s_issued[k] = issue_momentum<SG>(scn_of<ONE>(scns, one, tn.scn), maps, tn, smem + k * mom::stage_bytes<SG>(), &bar[k]);
    } else {
      s_issued[k] = 0;
    }
  };
  if (tid == 0) {
    for (int k = 0; k < NST; k++) mbar_init(&bar[k], 1);
    fence_barrier_init();
    s_stop = 0;
    for (int k = 0; k < NST - 1; k++) issue(tile + k * G, k);
  }
  uint32_t phase = 0u;  // bit s: parity of the next completion of stage s's barrier (a register, not a local array)
  // running CFL denominator of this thread's faces and the step scalars, for scenario cfl_st
  StepState* cfl_st = nullptr;
  StepVals sv{};
  CflTerms cfl;
  float cfl_dxinv = 0.0f, cfl_dyinv = 0.0f;
  int s = 0;  // stage of the current tile
  for (; tile < ntiles; tile += G) {
    const int sl = s == 0 ? NST - 1 : s - 1;  // stage of the previous tile, refilled now
    __syncthreads();  // s_issued[s] and s_tile[s] visible; stage sl no longer read
    if (tid == 0) {
      if (s_stop) {  // a wait of this CTA ran out: no further loads
        s_issued[sl] = 0;
      } else {
        fence_proxy_async();
        issue(tile + (NST - 1) * G, sl);
      }
    }
    if (s_issued[s]) {
      const Tile tl = s_tile[s];
      const ScnDev& S = scn_of<ONE>(scns, one, tl.scn);
      StepState& st = *S.st;
      if (&st != cfl_st) {  // the tile's scenario changed (CTA-uniform)
        flush_cfl(cfl_st, cfl, cfl_dxinv, cfl_dyinv, tx);
        cfl_st = &st;
        cfl = CflTerms{};
        cfl_dxinv = S.dxinv;
        cfl_dyinv = S.dyinv;
        sv = step_vals(st);
      }
      const bool ok = mbar_wait_bounded(&bar[s], (phase >> s) & 1u, S.wait_limit);
      phase ^= 1u << s;
      const int n = tl.n0 + tx, m = tl.m0 + ty;
      if (!ok) {
        st.fault = 1;
        s_stop = 1;
      } else if (n <= S.nmax && m <= S.mmax) {
        const unsigned char* sm = smem + s * mom::stage_bytes<SG>();
        const float* zs = (const float*)(sm + mom::O_ZS);
        const float* qu = (const float*)(sm + mom::O_QU);
        const float* qv = (const float*)(sm + mom::O_QV);
        const float* uu = (const float*)(sm + mom::O_UU);
        const float* vv = (const float*)(sm + mom::O_VV);
        auto ZS = [&](int dm, int dn) { return zs[(ty + dm) * mom::W_ZS + tx + dn]; };
        auto QU = [&](int dm, int dn) { return qu[(ty + 1 + dm) * mom::W_QU + tx + dn]; };
        auto QV = [&](int dm, int dn) { return qv[(ty + dm) * mom::W_QV + tx + 4 + dn]; };
        auto UU = [&](int dm, int dn) { return uu[(ty + 1 + dm) * mom::W_UV + tx + 4 + dn]; };
        auto VV = [&](int dm, int dn) { return vv[(ty + 1 + dm) * mom::W_UV + tx + 4 + dn]; };
        const uint16_t f = ((const uint16_t*)(sm + mom::O_FLAGS))[ty * 32 + tx];
        const uint8_t kfu = (sm + mom::O_KFU)[ty * 32 + tx];
        const uint8_t kfv = (sm + mom::O_KFV)[ty * 32 + tx];
        const int64_t c = (int64_t)m * S.ld + kGhostPad + n;
        const int p = sv.parity;
        const float zs_c = ZS(0, 0), zs_u = ZS(1, 0), zs_v = ZS(0, 1);
        const float zsu_u = fmaxf(zs_c, zs_u), zsu_v = fmaxf(zs_c, zs_v);
        float zmin_u, zmax_u = 0.0f, zmin_v, zmax_v = 0.0f;
        if (SG) {
          const float* gu = (const float*)(sm + mom::O_SGZU);
          const float* gv = (const float*)(sm + mom::O_SGZV);
          zmin_u = gu[ty * 64 + 2 * tx];
          zmax_u = gu[ty * 64 + 2 * tx + 1];
          zmin_v = gv[ty * 64 + 2 * tx];
          zmax_v = gv[ty * 64 + 2 * tx + 1];
        } else {
          zmin_u = ((const float*)(sm + mom::O_ZBMXU))[ty * 32 + tx];
          zmin_v = ((const float*)(sm + mom::O_ZBMXV))[ty * 32 + tx];
        }
        const bool act_u = f & F_UACT, act_v = f & F_VACT;
        const bool wet_u = act_u && (SG ? zsu_u > zmin_u + S.huthresh : zsu_u > zmin_u);
        const bool wet_v = act_v && (SG ? zsu_v > zmin_v + S.huthresh : zsu_v > zmin_v);
        // ---- issue the data-dependent table loads of both faces first
        SgLook lu{}, lv{};
        if (SG) {
          // A scattered read of one table record costs a whole 128-byte line of
          // DRAM traffic.  Each face keeps a cache entry: the 6 values it used
          // last step, contiguous per face, so a warp reads whole lines.  The
          // entry is requested first, its level code arrived with the tile, and
          // when the face still needs that level (water levels move slowly
          // against the table spacing) the entry is used; otherwise the tables
          // are read and the entry is refreshed.  Either way the values are the
          // table's, bit for bit.
          const int kc = ty * 32 + tx;
          auto look = [&](bool wet, float zsu, float zmin, float zmax, const float4* W, const UvRec* R, int o_rl,
                          float4* rc4, float2* rc2, uint8_t* rl, SgLook& L) {
            if (!wet) return;
            const float4 a = rc4[c];
            const float2 d = rc2[c];
            L.full = zsu > zmax;
            int code = kRecFull;
            const UvRec* r = nullptr;
            if (!L.full) {
              const SgLevel lv = sg_level(zsu, zmin, zmax, S.nlev);
              L.facint = lv.facint;
              r = R + (int64_t)(lv.iuv - 1) * S.nalloc + c;
              code = lv.iuv;
            }
            if (code == (int)(sm + o_rl)[kc]) {
              L.v = a;
              L.v2 = d;
            } else {
              if (L.full) {
                L.v = W[c];
                L.v2 = make_float2(0.0f, 0.0f);
              } else {
                L.v = *reinterpret_cast<const float4*>(r);
                L.v2 = *reinterpret_cast<const float2*>(&r->pwet);
              }
              rc4[c] = L.v;
              rc2[c] = L.v2;
              rl[c] = (uint8_t)code;
            }
          };
          look(wet_u, zsu_u, zmin_u, zmax_u, S.sgw_u, S.rec_u, mom::O_RLU, S.rc4_u, S.rc2_u, S.rl_u, lu);
          look(wet_v, zsu_v, zmin_v, zmax_v, S.sgw_v, S.rec_v, mom::O_RLV, S.rc4_v, S.rc2_v, S.rl_v, lv);
        }
        // ---- u face
        if (act_u) {
          float qn = 0.0f, un = 0.0f;
          if (wet_u) {
            FaceV a;
            a.qx_nm = QU(0, 0);
            a.qx_nmd = QU(-1, 0);
            a.qx_nmu = QU(1, 0);
            a.qy_nm = QV(0, 0);
            a.qy_nmu = QV(1, 0);
            a.qy_ndm = QV(0, -1);
            a.qy_ndmu = QV(1, -1);
            a.uu_nm = UU(0, 0);
            a.uu_nmd = UU(-1, 0);
            a.uu_nmu = UU(1, 0);
            a.uu_ndm = (f & F_CDN) ? UU(0, -1) : a.uu_nm;
            a.uu_num = (f & F_CUP) ? UU(0, 1) : a.uu_nm;
            a.vu = (VV(0, -1) + VV(1, -1) + VV(0, 0) + VV(1, 0)) / 4.0f;
            float hu, gnavg2, phi = 1.0f, zd0 = 0.0f, zd1 = 0.0f;
            bool dry0, dry1;
            if (SG) {
              const uint8_t* vn = sm + mom::O_VNEG;
              dry0 = vn[ty * 48 + tx] != 0;
              dry1 = vn[(ty + 1) * 48 + tx] != 0;
              if (S.wiggle) {
                const float* zd = (const float*)(sm + mom::O_ZSD);
                zd0 = zd[ty * mom::W_ZS + tx];
                zd1 = zd[(ty + 1) * mom::W_ZS + tx];
              }
              if (lu.full) {
                hu = lu.v.x + zsu_u;
                gnavg2 = sg_gnavg2_full(lu.v.z, lu.v.y, lu.v.w, zsu_u - zmax_u);
              } else {
                hu = fmaf(lu.v.y, lu.facint, lu.v.x);
                gnavg2 = fmaf(lu.v.w, lu.facint, lu.v.z);
                phi = fmaf(lu.v2.y, lu.facint, lu.v2.x);
              }
            } else {
              const float* zb = (const float*)(sm + mom::O_ZB);
              dry0 = zs_c < zb[ty * mom::W_ZS + tx];
              dry1 = zs_u < zb[(ty + 1) * mom::W_ZS + tx];
              hu = fmaxf(zsu_u - zmin_u, S.huthresh);
              gnavg2 = ((const float*)(sm + mom::O_GN2U))[ty * 32 + tx];
            }
            cfl.ghu_u = fmaxf(cfl.ghu_u, face_flux<SG, 0, MET>(S, sv, f, kfu, zs_c, zs_u, hu, gnavg2, phi, a, dry0, dry1,
                                                          zd0, zd1, c, qn, un));
            cfl.uv_u = fmaxf(cfl.uv_u, fabsf(un));
            S.qu[p ^ 1][c] = qn;
            S.uu[p ^ 1][c] = un;
          } else if (kfu & KF_WET2) {
            S.qu[p ^ 1][c] = 0.0f;
            S.uu[p ^ 1][c] = 0.0f;
          }
          const uint8_t kn = wet_u ? (uint8_t)(KF_WET | ((kfu & (KF_WET | KF_STALE)) ? KF_WET2 : 0))
                                   : (uint8_t)((kfu & (KF_WET | KF_STALE)) ? KF_WET2 : 0);
          if (kn != kfu) S.kf[0][c] = kn;
        }
        // ---- v face
        if (act_v) {
          float qn = 0.0f, un = 0.0f;
          if (wet_v) {
            FaceV a;
            a.qx_nm = QV(0, 0);
            a.qx_nmd = QV(0, -1);
            a.qx_nmu = QV(0, 1);
            a.qy_nm = QU(0, 0);
            a.qy_nmu = QU(0, 1);
            a.qy_ndm = QU(-1, 0);
            a.qy_ndmu = QU(-1, 1);
            a.uu_nm = VV(0, 0);
            a.uu_nmd = VV(0, -1);
            a.uu_nmu = VV(0, 1);
            a.uu_ndm = (f & F_CLF) ? VV(-1, 0) : a.uu_nm;
            a.uu_num = (f & F_CRT) ? VV(1, 0) : a.uu_nm;
            a.vu = (UU(-1, 0) + UU(-1, 1) + UU(0, 0) + UU(0, 1)) / 4.0f;
            float hu, gnavg2, phi = 1.0f, zd0 = 0.0f, zd1 = 0.0f;
            bool dry0, dry1;
            if (SG) {
              const uint8_t* vn = sm + mom::O_VNEG;
              dry0 = vn[ty * 48 + tx] != 0;
              dry1 = vn[ty * 48 + tx + 1] != 0;
              if (S.wiggle) {
                const float* zd = (const float*)(sm + mom::O_ZSD);
                zd0 = zd[ty * mom::W_ZS + tx];
                zd1 = zd[ty * mom::W_ZS + tx + 1];
              }
              if (lv.full) {
                hu = lv.v.x + zsu_v;
                gnavg2 = sg_gnavg2_full(lv.v.z, lv.v.y, lv.v.w, zsu_v - zmax_v);
              } else {
                hu = fmaf(lv.v.y, lv.facint, lv.v.x);
                gnavg2 = fmaf(lv.v.w, lv.facint, lv.v.z);
                phi = fmaf(lv.v2.y, lv.facint, lv.v2.x);
              }
            } else {
              const float* zb = (const float*)(sm + mom::O_ZB);
              dry0 = zs_c < zb[ty * mom::W_ZS + tx];
              dry1 = zs_v < zb[ty * mom::W_ZS + tx + 1];
              hu = fmaxf(zsu_v - zmin_v, S.huthresh);
              gnavg2 = ((const float*)(sm + mom::O_GN2V))[ty * 32 + tx];
            }
            cfl.ghu_v = fmaxf(cfl.ghu_v, face_flux<SG, 1, MET>(S, sv, f, kfv, zs_c, zs_v, hu, gnavg2, phi, a, dry0, dry1,
                                                          zd0, zd1, c, qn, un));
            cfl.uv_v = fmaxf(cfl.uv_v, fabsf(un));
            S.qv[p ^ 1][c] = qn;
            S.vv[p ^ 1][c] = un;
          } else if (kfv & KF_WET2) {
            S.qv[p ^ 1][c] = 0.0f;
            S.vv[p ^ 1][c] = 0.0f;
          }
          const uint8_t kn = wet_v ? (uint8_t)(KF_WET | ((kfv & (KF_WET | KF_STALE)) ? KF_WET2 : 0))
                                   : (uint8_t)((kfv & (KF_WET | KF_STALE)) ? KF_WET2 : 0);
          if (kn != kfv) S.kf[1][c] = kn;
        }
      }
    }
    s = s + 1 == NST ? 0 : s + 1;
  }
  flush_cfl(cfl_st, cfl, cfl_dxinv, cfl_dyinv, tx);
  if (tid == 0 && s_stop) drain_stages(bar, NST, phase);  // no copy in flight at exit
}

// --------------------------------------------------------------------------
// Continuity
// --------------------------------------------------------------------------
template <bool SG>
__device__ __forceinline__ bool issue_continuity(const ScnDev& S, const MapSet* maps, const Tile& tl,
                                                 unsigned char* st, uint64_t* bar) {
  const StepState& ss = *S.st;
  if (!ss.run) return false;
  const int p1 = ss.parity ^ 1;
  const int x = kGhostPad + tl.n0;
  const int y = tl.m0;
  uint32_t bytes = 32 * 9 * 4 + 36 * 8 * 4 + 32 * 8 * 4 * 2 + 32 * 8 * 2;
  if (SG) bytes += 32 * 8 * 8 + 32 * 8 * 4 + 32 * 8 + 32 * 8 + 2 * 32 * 8 * 4 + 32 * 8 * 8 + (S.wiggle ? 32 * 8 * 4 : 0);
  if (S.use_qext) bytes += 32 * 8 * 4;
  if (S.infiltration) bytes += 32 * 8 * 4 + (SG ? 0 : 32 * 8 * 4);
  mbar_expect_tx(bar, bytes);
  tma_load_2d(st + con::O_QU, map_of(maps, tl.scn, MC_QU0 + p1), x, y - 1, bar);
  tma_load_2d(st + con::O_QV, map_of(maps, tl.scn, MC_QV0 + p1), x - 4, y, bar);
  tma_load_2d(st + con::O_ZS, map_of(maps, tl.scn, MC_ZS), x, y, bar);
  tma_load_2d(st + con::O_ZSMAX, map_of(maps, tl.scn, MC_ZSMAX), x, y, bar);
  tma_load_2d(st + con::O_FLAGS, map_of(maps, tl.scn, MC_FLAGS), x, y, bar);
  if (SG) {
    tma_load_2d(st + con::O_ZVOL, map_of(maps, tl.scn, MC_ZVOL), x, y, bar);
    tma_load_2d(st + con::O_VOLMAX, map_of(maps, tl.scn, MC_VOLMAX), x, y, bar);
    tma_load_2d(st + con::O_VNEG, map_of(maps, tl.scn, MC_VNEG), x, y, bar);
    if (S.wiggle) tma_load_2d(st + con::O_ZS0, map_of(maps, tl.scn, MC_ZS0), x, y, bar);
    tma_load_2d(st + con::O_ZL, map_of(maps, tl.scn, MC_ZL), x, y, bar);
    tma_load_2d(st + con::O_ZZMIN, map_of(maps, tl.scn, MC_ZZMIN), x, y, bar);
    tma_load_2d(st + con::O_ZZMAX, map_of(maps, tl.scn, MC_ZZMAX), x, y, bar);
    tma_load_2d(st + con::O_ZC, map_of(maps, tl.scn, MC_ZC), 2 * x, y, bar);
  }
  if (S.use_qext) tma_load_2d(st + con::O_QEXT, map_of(maps, tl.scn, MC_QEXT), x, y, bar);
  if (S.infiltration) {
    tma_load_2d(st + con::O_QINF, map_of(maps, tl.scn, MC_QINF), x, y, bar);
    if (!SG) tma_load_2d(st + con::O_ZB, map_of(maps, tl.scn, MC_ZB), x, y, bar);
  }
  return true;
}

// EXT: the instance with the extended per-cell work (infiltration with
// state, cumulative sums, gridded rain, store variables); the plain instance
// keeps the register allocation of the common path.
template <bool SG, bool ONE, bool EXT>
__global__ void __launch_bounds__(256, 6) k_continuity_tma(const ScnDev* __restrict__ scns, const MapSet* __restrict__ maps,
                                                        const Tile* __restrict__ tiles, int ntiles,
                                                        const __grid_constant__ ScnDev one) {
  pdl_wait();  // the previous kernel of the step has completed
  pdl_trigger();
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_issued[2];
  __shared__ Tile s_tile[2];
  __shared__ int s_stop;  // a wait of this CTA ran out
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + 32 * ty;
  int tile = blockIdx.x;
  // thread 0: load tile t into stage k (the header travels to the other threads through shared memory)
  auto issue = [&](int t, int k) {
    if (t < ntiles) {
      const Tile tn = tiles[t];
      s_tile[k] = tn;
      s_issued[k] = issue_continuity<SG>(scn_of<ONE>(scns, one, tn.scn), maps, tn, smem + k * con::STAGE, &bar[k]);
    } else {
      s_issued[k] = 0;
    }
  };
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
    s_stop = 0;
    issue(tile, 0);
  }
  uint32_t phase = 0u;  // bit s: parity of the next completion of stage s's barrier (a register, not a local array)
  const StepState* sv_st = nullptr;  // scenario whose step scalars sv holds
  StepVals sv{};
  for (int it = 0; tile < ntiles; it++) {
    const int s = it & 1;
    const int next = tile + gridDim.x;
    __syncthreads();  // s_issued[s] and s_tile[s] visible; stage s^1 no longer read
    if (tid == 0) {
      if (s_stop) {  // a wait of this CTA ran out: no further loads
        s_issued[s ^ 1] = 0;
      } else {
        fence_proxy_async();
        issue(next, s ^ 1);
      }
    }
    if (s_issued[s]) {
      const Tile tl = s_tile[s];
      const ScnDev& S = scn_of<ONE>(scns, one, tl.scn);
      StepState& st = *S.st;
      if (&st != sv_st) {
        sv_st = &st;
        sv = step_vals(st);
      }
      const bool ok = mbar_wait_bounded(&bar[s], (phase >> s) & 1u, S.wait_limit);
      phase ^= 1u << s;
      const int n = tl.n0 + tx, m = tl.m0 + ty;
      if (!ok) {
        st.fault = 1;
        s_stop = 1;
      } else if (n <= S.nmax && m <= S.mmax) {
        const unsigned char* sm = smem + s * con::STAGE;
        const int k = ty * 32 + tx;
        const uint16_t f = ((const uint16_t*)(sm + con::O_FLAGS))[k];
        if (f & F_ACT) {
          const int64_t c = (int64_t)m * S.ld + kGhostPad + n;
          const float* qu = (const float*)(sm + con::O_QU);
          const float* qv = (const float*)(sm + con::O_QV);
          const float q_md = qu[ty * 32 + tx], q_mu = qu[(ty + 1) * 32 + tx];
          const float q_nd = qv[ty * 36 + tx + 3], q_nu = qv[ty * 36 + tx + 4];
          const float zs_old = ((const float*)(sm + con::O_ZS))[k];
          const float zm = ((const float*)(sm + con::O_ZSMAX))[k];
          const float dt = sv.dt;
          float zsn = zs_old;
          // infiltration with state (or cumulative rain) for every active cell, from the start-of-step state
          const bool inf_cell = EXT && S.precip && (S.inftype >= 2 || S.store_cumprcp);
          float qinf_cell = 0.0f;
          // rain of the cell: uniform from a time series, or from the gridded field
          float prc = sv.ptmp, netr = sv.ptmp;
          if (EXT && S.prcp_field) {
            const StepState& st0 = *S.st;
            const bool dry = SG ? ((const double*)(sm + con::O_ZVOL))[k] <= 0.0 : zs_old <= S.zb[c];
            prc = cell_rain(S, c, meteo_weights(S, st0.t, st0.meteo_t0, st0.meteo_t1), dry, netr);
          }
          if (inf_cell) {
            if (SG) {
              const double v0 = ((const double*)(sm + con::O_ZVOL))[k];
              qinf_cell = cell_infiltration(S, c, prc, dt, v0 <= 0.0, (float)(v0 / (double)S.area), S.st->ga_hs);
            } else {
              const float zbc = S.zb[c];
              qinf_cell = cell_infiltration(S, c, prc, dt, zs_old <= zbc, (float)((double)zs_old - (double)zbc),
                                            S.st->ga_hs);
            }
          }
          if (EXT && S.qinfmap)
            store_qinfmap(S, c, inf_cell, qinf_cell,
                          SG ? ((const double*)(sm + con::O_ZVOL))[k] > 0.0 : !(zs_old <= S.zb[c]));
          if (f & F_KCS1) {
            const float qx = S.use_qext ? ((const float*)(sm + con::O_QEXT))[k] : 0.0f;
            const float qi = S.infiltration ? ((const float*)(sm + con::O_QINF))[k] : 0.0f;
            if (SG) {
              const double v_old = ((const double*)(sm + con::O_ZVOL))[k];
              const float volmax = ((const float*)(sm + con::O_VOLMAX))[k];
              const uint8_t vn_old = (sm + con::O_VNEG)[k];
              const float zs00 = S.wiggle ? ((const float*)(sm + con::O_ZS0))[k] : 0.0f;
              float dvol = ((q_md - q_mu) * S.dy + (q_nd - q_nu) * S.dx) * dt;
              if (S.precip || S.use_qext) {
                float dzsdt = 0.0f;
                if (S.precip) {
                  const float qinfmap = inf_cell ? qinf_cell : ((S.infiltration && v_old > 0.0) ? qi : 0.0f);
                  dzsdt = dzsdt + (netr - qinfmap);
                }
                if (S.use_qext) dzsdt = dzsdt + qx;
                dvol = dvol + dzsdt * S.area * dt;
              }
              const double v = v_old + (double)dvol;
              if (v != v_old) S.zvol[c] = v;
              const float zs11 = zs_old;
              if (v >= (double)(volmax * 0.999f)) {
                zsn = (float)((double)fmaxf(((const float*)(sm + con::O_ZZMAX))[k], -20.0f) +
                              (v - (double)volmax) / (double)S.area);
              } else if (v <= (double)1.0e-6f) {
                zsn = fmaxf(((const float*)(sm + con::O_ZZMIN))[k], -20.0f);
              } else {
                const float dzvol = volmax / (float)(S.nlev - 1);
                const int iuv = lev_index(v / (double)dzvol, S.nlev);
                const float facint = (float)((v - (double)((float)(iuv - 1) * dzvol)) / (double)dzvol);
                // the cell's cached pair when it is still in interval iuv (a scattered
                // z_level read costs a whole 128-byte line), else the table's pair
                float2 dep;
                if (iuv == (int)(sm + con::O_ZL)[k]) {
                  dep = ((const float2*)(sm + con::O_ZC))[k];  // staged with the tile
                } else {
                  dep = S.zlev[(int64_t)(iuv - 1) * S.nalloc + c];
                  S.zc[c] = dep;
                  S.zl[c] = (uint8_t)iuv;
                }
                zsn = dep.x + dep.y * facint;
              }
              if (zsn != zs_old) S.zs[c] = zsn;
              if (S.wiggle) {
                if (zs11 != zs00) S.zs0[c] = zs11;
                S.zsderv[c] = zsn - 2.0f * zs11 + zs00;
              }
              const uint8_t vn = v < 0.0 ? 1 : 0;
              if (vn != vn_old) S.vneg[c] = vn;
            } else {
              float z = zs_old;
              if (S.precip) {
                const float zbc = S.infiltration ? ((const float*)(sm + con::O_ZB))[k] : 0.0f;
                const float qinfmap = inf_cell ? qinf_cell : ((S.infiltration && !(z <= zbc)) ? qi : 0.0f);
                z = z + (netr - qinfmap) * dt;
              }
              if (S.use_qext) z = z + qx * dt;
              z = z + ((q_md - q_mu) * S.dxinv + (q_nd - q_nu) * S.dyinv) * dt;
              if (z != zs_old) S.zs[c] = z;
              zsn = z;
            }
            if (EXT && (S.store_vmax | S.store_qmax | S.store_twet)) {
              float u_md = 0.0f, u_mu = 0.0f, u_nd = 0.0f, u_nu = 0.0f;
              if (S.store_vmax) {
                const int p1 = sv.parity ^ 1;  // this step's velocities
                u_md = S.uu[p1][c - S.ld];
                u_mu = S.uu[p1][c];
                u_nd = S.vv[p1][c - 1];
                u_nu = S.vv[p1][c];
              }
              store_cell_variables(S, c, q_md, q_mu, q_nd, q_nu, u_md, u_mu, u_nd, u_nu, zsn,
                                   S.store_twet ? (SG ? S.zz_min[c] : S.zb[c]) : 0.0f, dt);
            }
          }
          if (S.store_zsmax) {
            if (EXT && S.store_tzsmax) store_tzsmax(S, c, zsn, zm, SG ? S.zz_min[c] : S.zb[c]);
            if (zsn > zm) S.zsmax[c] = zsn;
          }
        }
      }
    }
    tile = next;
  }
  if (tid == 0 && s_stop) drain_stages(bar, 2, phase);  // no copy in flight at exit
}

// --------------------------------------------------------------------------
// Launchers
// --------------------------------------------------------------------------
int continuity_tma_smem() { return 2 * con::STAGE; }

// form: the momentum kernel variant, an autotuned choice: 4 / 5 compiled for
// 3 / 4 CTAs per SM (up to 80 / 64 registers per thread).  Both use two
// stages; three (loads issued two tiles ahead) measured slower on the 4M-cell
// subgrid workload.  one: the single scenario of the launch (passed by value),
// or null for an ensemble table.
int momentum_tma_smem(int form, int subgrid) { return 2 * (subgrid ? mom::STAGE_SG : mom::STAGE); }

template <bool SG, bool ONE, bool MET>
static const void* momentum_fn(int form) {
  return form == 5 ? (const void*)k_momentum_tma<SG, 4, ONE, 2, MET> : (const void*)k_momentum_tma<SG, 3, ONE, 2, MET>;
}
// form + 10: the instance with gridded wind / pressure fields
const void* momentum_tma_fn(int subgrid, int form, bool one) {
  const bool met = form >= 10;
  form = form % 10;
  if (met) {
    if (one) return subgrid ? momentum_fn<true, true, true>(form) : momentum_fn<false, true, true>(form);
    return subgrid ? momentum_fn<true, false, true>(form) : momentum_fn<false, false, true>(form);
  }
  if (one) return subgrid ? momentum_fn<true, true, false>(form) : momentum_fn<false, true, false>(form);
  return subgrid ? momentum_fn<true, false, false>(form) : momentum_fn<false, false, false>(form);
}
template <bool EXT>
static const void* continuity_fn(int subgrid, bool one) {
  if (one) return subgrid ? (const void*)k_continuity_tma<true, true, EXT> : (const void*)k_continuity_tma<false, true, EXT>;
  return subgrid ? (const void*)k_continuity_tma<true, false, EXT> : (const void*)k_continuity_tma<false, false, EXT>;
}
const void* continuity_tma_fn(int subgrid, bool one, bool ext) {
  return ext ? continuity_fn<true>(subgrid, one) : continuity_fn<false>(subgrid, one);
}

void launch_momentum_tma(const ScnDev* d_scns, const MapSet* d_maps, const Tile* d_tiles, int ntiles, int subgrid,
                         int form, int grid, cudaStream_t s, const ScnDev* one) {
  if (ntiles <= 0) return;
  static const ScnDev none{};
  // every form has this signature (ScnDev by value)
  using Kernel = void (*)(const ScnDev*, const MapSet*, const Tile*, int, ScnDev);
  const Kernel k = reinterpret_cast<Kernel>(const_cast<void*>(momentum_tma_fn(subgrid, form, one != nullptr)));
  launch_pdl(k, dim3(grid), dim3(32, 8), momentum_tma_smem(form, subgrid), s, d_scns, d_maps, d_tiles, ntiles,
             one ? *one : none);
}

void launch_continuity_tma(const ScnDev* d_scns, const MapSet* d_maps, const Tile* d_tiles, int ntiles, int subgrid,
                           int grid, cudaStream_t s, const ScnDev* one, bool ext) {
  if (ntiles <= 0) return;
  static const ScnDev none{};
  using Kernel = void (*)(const ScnDev*, const MapSet*, const Tile*, int, ScnDev);
  const Kernel k = reinterpret_cast<Kernel>(const_cast<void*>(continuity_tma_fn(subgrid, one != nullptr, ext)));
  launch_pdl(k, dim3(grid), dim3(32, 8), 2 * con::STAGE, s, d_scns, d_maps, d_tiles, ntiles, one ? *one : none);
}

}  // namespace sfg
