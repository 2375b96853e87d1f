// Data-interface kernels: gathers between the dense device layout and the
// reference's compacted cell order (nm), and a deterministic FP64 volume sum.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

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
__global__ void k_fill_f32(float* __restrict__ a, float v, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
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

// Volume of kcs==1 cells: subgrid sum(z_volume), regular sum((zs - zb) * cell area).
// Pass 1 writes one FP64 partial per CTA; pass 2 sums the partials in index
// order, so the result does not depend on scheduling.
__global__ void k_volume_partial(const ScnDev* __restrict__ scn, const int32_t* __restrict__ cmp, long long n,
                                 double* __restrict__ part) {
  const ScnDev& S = *scn;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int32_t c = cmp[i];
    if (!(S.flags[c] & F_KCS1)) continue;
    const float area = S.geo ? S.geo_area[c] : S.quadtree ? S.lv_area[S.qlev[c]] : S.area;
    acc += S.subgrid ? S.zvol[c] : ((double)S.zs[c] - (double)S.zb[c]) * (double)area;
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
void launch_fill_f32(float* a, float v, long long n, cudaStream_t s) {
  if (n > 0) k_fill_f32<<<grid_for(n), 256, 0, s>>>(a, v, n);
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

// ---- volume sum that allocates nothing ---------------------------------------
// launch_volume() above sums into buffers the model allocated when it was
// created.  Some callers want the volume at a moment when they must not
// allocate device memory at all: a server that reserved its whole HBM budget
// for resident models up front and admits work against that budget, or a
// host loop that cannot let a cudaMalloc/cudaFree synchronise the device while
// other models' steps are still running on other streams.  This variant keeps
// its scratch (one FP64 partial sum per CTA, then the total) in a fixed array
// compiled into the library, so a call performs no allocation of any kind.
//
// Limits: the array holds kNoAllocMaxParts partials.  The sum uses a
// grid-stride loop over at most that many CTAs, so every model size fits; a
// launch shape needing more partials is rejected with an error.  Nothing in
// the array has to start at zero: each CTA overwrites its own partial and the
// final pass overwrites the total before the host reads it.  There is one
// array per device, shared by every model on that device, so calls that
// overlap in time (two host threads, or two streams in flight) race on it and
// must be serialised by the caller.
constexpr int kNoAllocMaxParts = 4096;
static __device__ __align__(256) double g_volume_scratch[kNoAllocMaxParts + 1];  // partials, then the total

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};  // device address of g_volume_scratch, per device ordinal

// The first call on a device looks the array's address up with
// cudaGetSymbolAddress (with that device current); later calls reuse it.  Make
// the first call for each device before any stream capture begins.  The
// model's stream must belong to the current device: the address is only valid
// there.
int volume_scratch(cudaStream_t s, double** out, const char** why) {
  int dev = -1, sdev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    *why = "no usable current CUDA device for the volume scratch array";
    return 1;
  }
  if (cudaStreamGetDevice(s, &sdev) != cudaSuccess || sdev != dev) {
    *why = "the model's stream is not on the current CUDA device; make the model's device current first";
    return 1;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_volume_scratch);
    if (e != cudaSuccess || !p) {
      *why = "cudaGetSymbolAddress failed for the volume scratch array";
      return 1;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return 0;
}
}  // namespace

// Same sum as launch_volume (same kernels, same launch shape, so the same
// bits), with the partials and the total in g_volume_scratch; the total is
// copied to *host_out and the stream is synchronised before returning.
int volume_noalloc(const ScnDev* d_scn, const int32_t* cmp, long long n, cudaStream_t s, double* host_out,
                   const char** why) {
  if (n < 0) {
    *why = "negative cell count";
    return 1;
  }
  const int g = grid_for(n);
  if (g > kNoAllocMaxParts) {
    *why = "volume sum needs more partial sums than the fixed scratch array holds (4096)";
    return 1;
  }
  double* scratch = nullptr;
  if (volume_scratch(s, &scratch, why)) return 1;
  // an error left by an earlier, unrelated call is reported as such, not as a launch failure here
  if (cudaPeekAtLastError() != cudaSuccess) {
    *why = "an earlier CUDA error is still pending on this thread";
    return 1;
  }
  k_volume_partial<<<g, 256, 0, s>>>(d_scn, cmp, n, scratch);
  if (cudaGetLastError() != cudaSuccess) {
    *why = "volume partial-sum kernel launch failed";
    return 1;
  }
  k_volume_final<<<1, 32, 0, s>>>(scratch, g, scratch + kNoAllocMaxParts);
  if (cudaGetLastError() != cudaSuccess) {
    *why = "volume final-sum kernel launch failed";
    return 1;
  }
  if (cudaMemcpyAsync(host_out, scratch + kNoAllocMaxParts, sizeof(double), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    *why = "copy of the volume to the host failed";
    return 1;
  }
  return 0;
}

}  // namespace sfg
