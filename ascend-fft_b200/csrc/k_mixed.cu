// Mixed-radix C2C for 7-smooth lengths (n = 2^a 3^b 5^c 7^d up to kMixedMaxN), one HBM pass.
// Stockham autosort: pass p of radix R over Ns = R_0 ... R_(p-1) takes butterfly j < n/R,
// k = j mod Ns, inputs x[j + r n/R], twiddles W_(Ns R)^(k r) = W_n^(k r n/(Ns R)) (one FP64-built
// table of W_n^m, m < n, indexed without a modulo since k r n/(Ns R) < n), an R-point DFT in
// registers and outputs at (j - k) R + k + r Ns.  A row of n values lives in two shared buffers
// (ping-pong); the first pass reads HBM directly (coalesced over j), the last writes HBM
// directly (Ns = n/R there, so the store index is j + r n/R, coalesced too).  T = ceil(n/8)
// threads per row, each taking butterflies j = t, t + T, ...; rows packed to ~256 threads.
// The radix list is a kernel argument, so one kernel serves every such length.
#include <cuda_runtime.h>

#include <algorithm>

#include "backend.h"
#include "fft_kernels.cuh"
#include "fft_odd.cuh"

namespace bfly {
namespace dev {

struct MixedArgs {
    int n, passes;
    int radix[backend::kMixedMaxPasses];
    int ns[backend::kMixedMaxPasses];
};

// KIND bit 0: source is the row in HBM; bit 1: destination is the row in HBM (scaled).
template <int R, bool INV, int KIND>
__device__ __forceinline__ void mixed_pass(const float2* __restrict__ src, float2* __restrict__ dst, int n, int Ns,
                                           const float2* __restrict__ tw, int t, int T, float scale) {
    const int nb = n / R;
    const int tws = n / (Ns * R);
    for (int j = t; j < nb; j += T) {
        const int k = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = (KIND & 1) ? ld_stream(src + j + r * nb) : src[spad(j + r * nb)];
        if (k) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul<INV>(v[r], __ldg(tw + k * r * tws));
        }
        DFT<R, INV>::run(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (KIND & 2) st_stream(dst + base + r * Ns, cscale(v[r], scale));
            else dst[spad(base + r * Ns)] = v[r];
        }
    }
}

template <bool INV, int KIND>
__device__ __forceinline__ void mixed_pass_r(int R, const float2* src, float2* dst, int n, int Ns, const float2* tw,
                                             int t, int T, float scale) {
    switch (R) {
        case 16: mixed_pass<16, INV, KIND>(src, dst, n, Ns, tw, t, T, scale); break;
        case 8: mixed_pass<8, INV, KIND>(src, dst, n, Ns, tw, t, T, scale); break;
        case 4: mixed_pass<4, INV, KIND>(src, dst, n, Ns, tw, t, T, scale); break;
        case 2: mixed_pass<2, INV, KIND>(src, dst, n, Ns, tw, t, T, scale); break;
        case 7: mixed_pass<7, INV, KIND>(src, dst, n, Ns, tw, t, T, scale); break;
        case 5: mixed_pass<5, INV, KIND>(src, dst, n, Ns, tw, t, T, scale); break;
        default: mixed_pass<3, INV, KIND>(src, dst, n, Ns, tw, t, T, scale); break;
    }
}

template <bool INV>
__global__ void __launch_bounds__(1024) k_mixed(const float2* __restrict__ in, float2* __restrict__ out,
                                                const float2* __restrict__ tw, MixedArgs a, uint64_t batch, int T,
                                                int rows, int len, float scale) {
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * rows + rl;
    const bool ok = rl < rows && row < batch;
    const int n = a.n;
    const float2* src = in + row * n;
    float2* dst = out + row * n;
    float2* buf0 = smem + (size_t)(rl < rows ? rl : 0) * 2 * len;
    float2* buf1 = buf0 + len;
    for (int p = 0; p < a.passes; ++p) {
        const int R = a.radix[p], Ns = a.ns[p];
        const bool first = p == 0, last = p == a.passes - 1;
        const float2* s = (p & 1) ? buf0 : buf1;   // written by pass p - 1
        float2* d = (p & 1) ? buf1 : buf0;
        if (ok) {
            if (first && last) mixed_pass_r<INV, 3>(R, src, dst, n, Ns, tw, t, T, scale);
            else if (first) mixed_pass_r<INV, 1>(R, src, d, n, Ns, tw, t, T, scale);
            else if (last) mixed_pass_r<INV, 2>(R, s, dst, n, Ns, tw, t, T, scale);
            else mixed_pass_r<INV, 0>(R, s, d, n, Ns, tw, t, T, scale);
        }
        if (!last) __syncthreads();
    }
}

}  // namespace dev

namespace backend {

int launchMixed(const void* in, void* out, const MixedRadix& plan, uint64_t batch, bool inverse, float scale,
                const void* tw, void* stream) {
    if (plan.n < 2 || plan.passes < 1 || plan.passes > kMixedMaxPasses || (uint32_t)plan.n > kMixedMaxN)
        return (int)cudaErrorInvalidValue;
    dev::MixedArgs a;
    a.n = plan.n;
    a.passes = plan.passes;
    for (int p = 0; p < kMixedMaxPasses; ++p) {
        a.radix[p] = plan.radix[p];
        a.ns[p] = plan.ns[p];
    }
    const int T = std::min(1024, (plan.n + 7) / 8);
    const int rows = std::max(1, 256 / T);
    const int len = dev::spad(plan.n - 1) + 1;
    const int smem = rows * 2 * len * 8;
    auto* fn = inverse ? dev::k_mixed<true> : dev::k_mixed<false>;
    // opted in once per device at the largest row pair (n = kMixedMaxN, one row per CTA)
    constexpr int kMaxSmem = 2 * (dev::spad((int)kMixedMaxN - 1) + 1) * 8;
    static_assert(kMaxSmem <= 227 * 1024, "two rows of the longest length fit in shared memory");
    if (smem > kMaxSmem) return (int)cudaErrorInvalidValue;
    if (int e = optInSharedMemory((const void*)fn, kMaxSmem)) return e;
    const uint64_t grid = (batch + rows - 1) / rows;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, T * rows, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw), a, batch, T, rows,
        len, scale);
    return (int)cudaGetLastError();
}

}  // namespace backend
}  // namespace bfly
