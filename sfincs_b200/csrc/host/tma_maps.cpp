// TMA tensor maps of a scenario's dense arrays (2-D: ld columns x (mmax+2) rows).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstring>
#include <stdexcept>
#include <string>

#include "model.h"

namespace sfg {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    check_cuda(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q), "driver entry point");
    if (q != cudaDriverEntryPointSuccess || !p) throw std::runtime_error("cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// width/rows in elements, row_bytes = row pitch; box (bw x bh) elements.
void encode(unsigned char* out, CUtensorMapDataType type, const void* base, uint64_t width, uint64_t rows,
            uint64_t row_bytes, uint32_t bw, uint32_t bh, const char* what) {
  std::memset(out, 0, 128);
  if (!base) return;  // array not allocated for this model: the kernels never issue its load
  cuuint64_t dims[2] = {width, rows};
  cuuint64_t strides[1] = {row_bytes};
  cuuint32_t box[2] = {bw, bh};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(reinterpret_cast<CUtensorMap*>(out), type, 2, const_cast<void*>(base), dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error(std::string("cuTensorMapEncodeTiled failed for ") + what);
}

}  // namespace

MapSet build_map_set(const ScnDev& d) {
  MapSet ms;
  std::memset(&ms, 0, sizeof(ms));
  const uint64_t W = (uint64_t)d.ld, R = (uint64_t)(d.mmax + 2);
  auto f32 = [&](int id, const void* p, uint32_t bw, uint32_t bh, const char* nm) {
    encode(ms.m[id], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p, W, R, W * 4, bw, bh, nm);
  };
  // momentum boxes (32 x 8 tiles; halos as laid out in kernels_tma.cu)
  f32(MM_ZS, d.zs, 36, 9, "zs");
  for (int b = 0; b < 2; b++) {
    f32(MM_QU0 + b, d.qu[b], 36, 10, "qu");
    f32(MM_QV0 + b, d.qv[b], 40, 9, "qv");
    f32(MM_UU0 + b, d.uu[b], 40, 10, "uu");
    f32(MM_VV0 + b, d.vv[b], 40, 10, "vv");
  }
  encode(ms.m[MM_FLAGS], CU_TENSOR_MAP_DATA_TYPE_UINT16, d.flags, W, R, W * 2, 32, 8, "flags");
  encode(ms.m[MM_KFU], CU_TENSOR_MAP_DATA_TYPE_UINT8, d.kf[0], W, R, W, 32, 8, "kfu");
  encode(ms.m[MM_KFV], CU_TENSOR_MAP_DATA_TYPE_UINT8, d.kf[1], W, R, W, 32, 8, "kfv");
  if (d.subgrid) {
    encode(ms.m[MM_VNEG], CU_TENSOR_MAP_DATA_TYPE_UINT8, d.vneg, W, R, W, 48, 9, "vneg");
    if (d.wiggle) f32(MM_ZSD, d.zsderv, 36, 9, "zsderv");
    encode(ms.m[MM_SGZU], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, d.sgz_u, 2 * W, R, 2 * W * 4, 64, 8, "sgz_u");
    encode(ms.m[MM_SGZV], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, d.sgz_v, 2 * W, R, 2 * W * 4, 64, 8, "sgz_v");
    // record-cache codes (one byte per face)
    encode(ms.m[MM_RLU], CU_TENSOR_MAP_DATA_TYPE_UINT8, d.rl_u, W, R, W, 32, 8, "record codes u");
    encode(ms.m[MM_RLV], CU_TENSOR_MAP_DATA_TYPE_UINT8, d.rl_v, W, R, W, 32, 8, "record codes v");
  } else {
    f32(MM_ZB, d.zb, 36, 9, "zb");
    f32(MM_ZBMXU, d.zbmx_u, 32, 8, "zbmx_u");
    f32(MM_ZBMXV, d.zbmx_v, 32, 8, "zbmx_v");
    f32(MM_GN2U, d.gn2_u, 32, 8, "gn2_u");
    f32(MM_GN2V, d.gn2_v, 32, 8, "gn2_v");
  }
  // continuity boxes
  for (int b = 0; b < 2; b++) {
    f32(MC_QU0 + b, d.qu[b], 32, 9, "qu (continuity)");
    f32(MC_QV0 + b, d.qv[b], 36, 8, "qv (continuity)");
  }
  f32(MC_ZS, d.zs, 32, 8, "zs (continuity)");
  f32(MC_ZSMAX, d.zsmax, 32, 8, "zsmax");
  encode(ms.m[MC_FLAGS], CU_TENSOR_MAP_DATA_TYPE_UINT16, d.flags, W, R, W * 2, 32, 8, "flags (continuity)");
  if (d.subgrid) {
    encode(ms.m[MC_ZVOL], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, d.zvol, W, R, W * 8, 32, 8, "z_volume");
    f32(MC_VOLMAX, d.zz_volmax, 32, 8, "z_volmax");
    encode(ms.m[MC_VNEG], CU_TENSOR_MAP_DATA_TYPE_UINT8, d.vneg, W, R, W, 32, 8, "vneg (continuity)");
    if (d.wiggle) f32(MC_ZS0, d.zs0, 32, 8, "zs0");
    encode(ms.m[MC_ZL], CU_TENSOR_MAP_DATA_TYPE_UINT8, d.zl, W, R, W, 32, 8, "z_level cache codes");
    f32(MC_ZZMIN, d.zz_min, 32, 8, "z_zmin");
    f32(MC_ZZMAX, d.zz_max, 32, 8, "z_zmax");
    encode(ms.m[MC_ZC], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, d.zc, 2 * W, R, 2 * W * 4, 64, 8, "z_level cache");
  }
  if (d.use_qext) f32(MC_QEXT, d.qext, 32, 8, "qext");
  if (d.infiltration) {
    f32(MC_QINF, d.qinf, 32, 8, "qinf");
    if (!d.subgrid) f32(MC_ZB, d.zb, 32, 8, "zb (continuity)");
  }
  return ms;
}

}  // namespace sfg
