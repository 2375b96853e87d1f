// Data-interface kernels: gathers between the dense device layout and the
// reference's compacted cell order (nm), and a deterministic FP64 volume sum.
#include <cuda_runtime.h>

#include <cstdint>

#include "sfg_device.h"

namespace sfg {

__global__ void k_gather_f32_f64(const float* __restrict__ src, const int32_t* __restrict__ cmp,
                                 double* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (double)src[cmp[i]];
}
__global__ void k_gather_f32(const float* __restrict__ src, const int32_t* __restrict__ cmp, float* __restrict__ out,
                             long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = src[cmp[i]];
}
__global__ void k_gather_f64(const double* __restrict__ src, const int32_t* __restrict__ cmp, double* __restrict__ out,
                             long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = src[cmp[i]];
}
// Wet flags (bit 0) of the u and v face of every cell: out[0:n] = u, out[n:2n] = v.
__global__ void k_gather_u8(const uint8_t* __restrict__ ku, const uint8_t* __restrict__ kv,
                            const int32_t* __restrict__ cmp, float* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    out[i] = (float)(ku[cmp[i]] & 1);
    out[n + i] = (float)(kv[cmp[i]] & 1);
  }
}
__global__ void k_or_u8(uint8_t* __restrict__ a, uint8_t mask, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] |= mask;
}
__global__ void k_scatter_f32(const float* __restrict__ in, const int32_t* __restrict__ cmp, float* __restrict__ dst,
                              long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[cmp[i]] = in[i];
}
__global__ void k_scatter_f64_f32(const double* __restrict__ in, const int32_t* __restrict__ cmp,
                                  float* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[cmp[i]] = (float)in[i];
}

// Volume of kcs==1 cells: subgrid sum(z_volume), regular sum((zs - zb) * area).
// Pass 1 writes one FP64 partial per CTA; pass 2 sums the partials in index
// order, so the result does not depend on scheduling.
__global__ void k_volume_partial(const ScnDev* __restrict__ scn, const int32_t* __restrict__ cmp, long long n,
                                 double* __restrict__ part) {
  const ScnDev& S = *scn;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int32_t c = cmp[i];
    if (!(S.flags[c] & F_KCS1)) continue;
    acc += S.subgrid ? S.zvol[c] : ((double)S.zs[c] - (double)S.zb[c]) * (double)S.area;
  }
  __shared__ double s[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s[w];
    part[blockIdx.x] = t;
  }
}
__global__ void k_volume_final(const double* __restrict__ part, int nparts, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < nparts; i++) t += part[i];
    *out = t;
  }
}

static int grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

void launch_gather_f32_f64(const float* src, const int32_t* cmp, double* out, long long n, cudaStream_t s) {
  if (n > 0) k_gather_f32_f64<<<grid_for(n), 256, 0, s>>>(src, cmp, out, n);
}
void launch_gather_f32(const float* src, const int32_t* cmp, float* out, long long n, cudaStream_t s) {
  if (n > 0) k_gather_f32<<<grid_for(n), 256, 0, s>>>(src, cmp, out, n);
}
void launch_gather_f64(const double* src, const int32_t* cmp, double* out, long long n, cudaStream_t s) {
  if (n > 0) k_gather_f64<<<grid_for(n), 256, 0, s>>>(src, cmp, out, n);
}
void launch_gather_u8(const uint8_t* ku, const uint8_t* kv, const int32_t* cmp, float* out, long long n,
                      cudaStream_t s) {
  if (n > 0) k_gather_u8<<<grid_for(n), 256, 0, s>>>(ku, kv, cmp, out, n);
}
void launch_or_u8(uint8_t* a, uint8_t mask, long long n, cudaStream_t s) {
  if (n > 0) k_or_u8<<<grid_for(n), 256, 0, s>>>(a, mask, n);
}
void launch_scatter_f32(const float* in, const int32_t* cmp, float* dst, long long n, cudaStream_t s) {
  if (n > 0) k_scatter_f32<<<grid_for(n), 256, 0, s>>>(in, cmp, dst, n);
}
void launch_scatter_f64_f32(const double* in, const int32_t* cmp, float* dst, long long n, cudaStream_t s) {
  if (n > 0) k_scatter_f64_f32<<<grid_for(n), 256, 0, s>>>(in, cmp, dst, n);
}
int volume_parts(long long n) { return grid_for(n); }
void launch_volume(const ScnDev* d_scn, const int32_t* cmp, long long n, double* part, double* out, cudaStream_t s) {
  const int g = grid_for(n);
  k_volume_partial<<<g, 256, 0, s>>>(d_scn, cmp, n, part);
  k_volume_final<<<1, 32, 0, s>>>(part, g, out);
}

}  // namespace sfg
