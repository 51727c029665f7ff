// Programmatic dependent launch (PDL).
//
// A launch with cudaLaunchAttributeProgrammaticStreamSerialization may be
// scheduled while the kernel before it in the stream drains.  Every kernel
// launched that way begins with pdl_wait() (griddepcontrol.wait: the stream's
// previous kernel has completed and its memory is visible) before it touches
// global memory, and calls pdl_trigger() (griddepcontrol.launch_dependents)
// where the next launch may be scheduled: its CTAs take the SM slots this
// grid leaves and wait the same way.  Without the attribute both
// instructions return at once, and a predecessor without the trigger simply
// completes first, so other kernels in the stream need nothing of it.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace nttb {

__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
__device__ __forceinline__ void pdl_trigger() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}
// wait, then let the next launch be scheduled at once
__device__ __forceinline__ void pdl_enter() {
    pdl_wait();
    pdl_trigger();
}

// Launch `kernel` (which starts with pdl_wait) with the PDL attribute.
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = grid;
    lc.blockDim = block;
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, kernel, std::forward<Args>(args)...);
}

}  // namespace nttb
