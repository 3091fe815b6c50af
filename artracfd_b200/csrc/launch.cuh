// Kernel launch with programmatic dependent launch (PDL).
//
// A kernel launched through launch_k may be scheduled while the kernel before
// it on the stream drains (and, in a captured CUDA graph, the edge between
// them becomes a programmatic one), which hides most of the launch gap of the
// short kernels of a time step.  Every kernel launched this way calls
// pdl_wait() before its first access to memory that an earlier kernel
// writes: griddepcontrol.wait returns once the preceding grid has completed
// and its writes are visible, and is a no-op for a kernel launched without
// the attribute.  No kernel triggers its dependents early, so the order of
// the stream is kept.  ACFD_PDL=0 in the environment launches without it.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace acfd {

bool pdl_enabled();

__device__ __forceinline__ void pdl_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace acfd
