// pdl.cuh -- programmatic dependent launch (sm_90 and later).
//
// A kernel launched with launchDependent() may be scheduled while the
// previous kernel of its stream (or the graph node it depends on) is still
// running.  Every such kernel calls gridDependencyWait() before its first
// global memory access: the instruction returns once the previous grid has
// completed and its writes are visible, so the kernel sees exactly what it
// would see after an ordinary launch.  gridDependentsLaunch() then lets the
// next kernel of the stream be scheduled early in turn.  What the overlap
// removes is the launch gap between short dependent kernels; for a kernel
// launched the ordinary way both instructions do nothing.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace vfb
{
__device__ __forceinline__ void gridDependencyWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void gridDependentsLaunch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// kernel<<<grid, block, smem, stream>>>(args...) with programmatic stream
// serialisation allowed
template <class... P, class... A>
cudaError_t launchDependent(void (*kernel)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t stream,
                            A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}
} // namespace vfb
