// Programmatic dependent launch (sm_90 and later), used inside the three kernels of a power-of-two product
// (the x-mix and the y-inverse are launched as dependents): a kernel launched with the programmatic
// stream-serialisation attribute may be scheduled while its predecessor on the stream is still running;
// its CTAs then block in griddep_wait() until the predecessor has completed and its memory is visible.
// Each kernel launched this way calls griddep_wait() before anything else (so it reads no data of its
// predecessor early) and griddep_launch_dependents() right after, so that its own successor may be
// scheduled as its CTAs retire. Outside such a launch both instructions do nothing.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace rtm {

__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                    Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace rtm
