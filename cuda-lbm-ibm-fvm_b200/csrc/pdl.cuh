// pdl.cuh -- programmatic dependent launch for the library's kernels.
//
// A kernel launched by pdl_launch carries
// cudaLaunchAttributeProgrammaticStreamSerialization: it may be scheduled
// while the grid before it in the stream is still finishing.  Every such
// kernel begins with pdl_enter(): it waits for that grid to complete (and its
// writes to be visible) before its first global memory access, then lets the
// grid after it launch.  The launch and prologue of a kernel so overlap the
// end of the one before; results are those of ordinary stream order.
// Launched without the attribute, the wait returns at once.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace vof {

__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
static inline cudaError_t pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                     cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace vof
