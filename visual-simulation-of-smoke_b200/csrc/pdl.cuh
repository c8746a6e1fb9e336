// Programmatic dependent launch, shared by the step, multigrid and network kernels.
//
// A kernel launched with launch_pdl (programmatic stream serialisation) may start while the stream's previous kernel
// is still running: its blocks are dispatched as soon as every block of the previous kernel has called pdl_trigger
// (or exited). So the launch and the block dispatch overlap the previous kernel's tail. Every kernel launched this way
// calls pdl_wait before it reads anything a previous kernel writes and before it writes any global memory; the wait
// returns once the previous kernel has completed and its writes are visible. A kernel that waits before it completes
// makes the chain transitive, so each kernel sees every earlier kernel's results. Without the launch attribute the
// wait returns at once.
#pragma once

#include <utility>

#include <cuda_runtime.h>

namespace smoke_b200 {

#ifdef __CUDACC__
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Both, at the top of a kernel that reads its inputs right away.
__device__ __forceinline__ void pdl_begin() {
    pdl_trigger();
    pdl_wait();
}

template <typename... P, typename... A>
inline void launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}
#endif

}  // namespace smoke_b200
