// Programmatic dependent launch (PDL) helpers shared by the step kernels.
//
// The kernels of a step are launched so that the next one may start while the previous one
// runs. Each waits for its predecessor (grid completion and memory) before it reads what the
// predecessor wrote or writes what the predecessor reads. A grid completes only after its own
// wait returned, so waiting on the predecessor's completion also covers every grid before it.
// Most kernels let their dependents launch right after that wait; the batched epilogue
// (mixed_rows) does so at its start, since everything the next GEMM does before its own wait
// (barriers, tensor memory, static G tiles) touches nothing the epilogue reads or writes.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace dtb {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
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

}  // namespace dtb
