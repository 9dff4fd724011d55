/* Programmatic dependent launch (CUDA 12.3+, recorded by stream capture into graphs).
 *
 * launch_dep launches a kernel with cudaLaunchAttributeProgrammaticStreamSerialization when the
 * context allows it (GAT_TUNE_DEP_LAUNCH, on by default): the GPU may then set the kernel up
 * while the previous kernel of the stream finishes. No kernel here triggers its dependents
 * early, so a dependent grid starts only after every block of the previous grid has exited.
 * Every kernel launched this way calls dep_wait() first, which returns once the previous grid
 * has completed and its writes are visible; ordering in the stream is therefore the same as
 * without the attribute, minus the launch gap. dep_wait() is a no-op for a kernel launched
 * without the attribute. */
#pragma once

#include <mutex>
#include <set>
#include <utility>

#include "internal.h"

namespace gat {

__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

/* Sets a kernel's preferred split between L1 and shared memory (percent of the largest shared
 * size) the first time it is asked for on a device; later requests for the same kernel keep the
 * first value. An SM takes the split of the first block that lands on it while it is empty and
 * keeps it until it is empty again, so a long-running kernel fixes the split of its SMs for every
 * other stream's blocks. */
inline void prefer_split(const void* kernel, int device, int pct) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    std::lock_guard<std::mutex> lk(mu);
    if (!done.insert({kernel, device}).second) return;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct) != cudaSuccess)
        cudaGetLastError();
}

template <class... P, class... A>
inline cudaError_t launch_dep(const gat_ctx* ctx, void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, A&&... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = ctx->dep_launch ? 1 : 0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

/* zeroes n ints in stream order (a kernel, so a chain of dependent launches stays unbroken) */
__global__ void k_zero_words(int* p, int n);

}  // namespace gat
