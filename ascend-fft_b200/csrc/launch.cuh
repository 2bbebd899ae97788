// Kernel launch with programmatic stream serialisation (programmatic dependent launch): the
// kernel may begin launching while the previous kernel on the stream drains; kernels launched
// this way call pdl_trigger() and pdl_wait() (fft_core.cuh) before their first global access.
// BFLY_PDL=0 in the environment launches them plainly instead (read once per process).
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>

namespace bfly {
namespace backend {

inline bool pdlEnabled() {
    static const bool on = [] {
        const char* env = std::getenv("BFLY_PDL");
        return !(env && env[0] == '0');
    }();
    return on;
}

// `args` must have exactly the kernel's parameter types.
template <typename... Args>
cudaError_t launchPdl(const void* fn, unsigned grid, int block, int smem, cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdlEnabled() ? 1 : 0;
    void* argv[] = {static_cast<void*>(&args)...};
    return cudaLaunchKernelExC(&cfg, fn, argv);
}

}  // namespace backend
}  // namespace bfly
