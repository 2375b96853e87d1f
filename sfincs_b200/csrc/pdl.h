// Programmatic dependent launch (sm_90+): the kernels of a time step are
// launched with the programmatic-stream-serialization attribute, so the next
// kernel's CTAs can be scheduled while the current one drains instead of
// after a full launch gap.  Every such kernel calls pdl_wait() before it
// reads or writes anything the previous kernel touches; the wait returns once
// that kernel has completed and its memory is visible.  pdl_trigger() lets
// the dependent launch as soon as every CTA of this kernel has reached it.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace sfg {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace sfg
