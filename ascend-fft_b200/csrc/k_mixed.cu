// Mixed-radix C2C for 13-smooth lengths (n = 2^a 3^b 5^c 7^d 11^e 13^f up to kMixedMaxN), one
// HBM pass.
// Stockham autosort: pass p of radix R over Ns = R_0 ... R_(p-1) takes butterfly j < n/R,
// k = j mod Ns, inputs x[j + r n/R], twiddles W_(Ns R)^(k r) from the pass's slice of an
// FP64-built table (entry (r-1) Ns + k: consecutive threads read consecutive entries), an
// R-point DFT in registers (radix 2..16, odd and Good-Thomas composite radices included) and
// outputs at (j - k) R + k + r Ns.  A row of n values lives in two shared buffers (ping-pong);
// the first pass reads HBM directly (coalesced over j), the last writes HBM directly (Ns = n/R
// there, so the store index is j + r n/R, coalesced too).  T = min(512, ceil(n / R_max)) threads
// per row, each taking butterflies j = t, t + T, ...; max(1, 224 / T) rows per CTA.  k = j mod Ns
// uses a multiply-high by ceil(2^32 / Ns) (exact for j, Ns < 2^14).  The pass list is a kernel
// argument, so one kernel serves every such length.
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
    int twoff[backend::kMixedMaxPasses];
    unsigned magic[backend::kMixedMaxPasses];   // ceil(2^32 / ns), pass p >= 1
    int pad0;          // the buffer pass 0 writes: element i at i + i / pad0 (pad0 = 0: at i)
    unsigned magic0;   // ceil(2^32 / pad0)
};

// Shared-memory position of element i: the buffer pass 0 writes is padded by one slot every
// pad0 elements (pad0 = R_0 when even, so its stride-R_0 stores hit distinct banks); the
// others use spad.
template <bool PASS0_BUF>
__device__ __forceinline__ int mixed_at(int i, int pad0, unsigned magic0) {
    if constexpr (PASS0_BUF) return pad0 ? i + (int)__umulhi((unsigned)i, magic0) : i;
    else return spad(i);
}

// KIND bit 0: source is the row in HBM (pass 0, which writes the pass-0 buffer); bit 1:
// destination is the row in HBM (scaled); bit 2: source is the pass-0 buffer (pass 1).
// Pass 0 (Ns = 1) has no twiddles.
template <int R, bool INV, int KIND>
__device__ __forceinline__ void mixed_pass(const float2* __restrict__ src, float2* __restrict__ dst, int n, int Ns,
                                           unsigned magic, const float2* __restrict__ twp, int t, int T,
                                           float scale, int pad0, unsigned magic0) {
    const int nb = n / R;
    for (int j = t; j < nb; j += T) {
        const int k = (KIND & 1) ? 0 : j - Ns * (int)__umulhi((unsigned)j, magic);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
            v[r] = (KIND & 1) ? ld_stream(src + j + r * nb) : src[mixed_at<(KIND & 4) != 0>(j + r * nb, pad0, magic0)];
        if (!(KIND & 1)) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul<INV>(v[r], __ldg(twp + (r - 1) * Ns + k));
        }
        DFT<R, INV>::run(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (KIND & 2) st_stream(dst + base + r * Ns, cscale(v[r], scale));
            else dst[mixed_at<(KIND & 1) != 0>(base + r * Ns, pad0, magic0)] = v[r];
        }
    }
}

// WIDE adds the prime radices 11 and 13 (their butterflies need more registers, so plans
// without them run an instance compiled without those cases).
template <bool INV, int KIND, bool WIDE>
__device__ __forceinline__ void mixed_pass_r(int R, const float2* src, float2* dst, int n, int Ns, unsigned magic,
                                             const float2* twp, int t, int T, float scale, int pad0,
                                             unsigned magic0) {
    if constexpr (WIDE) {
        if (R == 13) return mixed_pass<13, INV, KIND>(src, dst, n, Ns, magic, twp, t, T, scale, pad0, magic0);
        if (R == 11) return mixed_pass<11, INV, KIND>(src, dst, n, Ns, magic, twp, t, T, scale, pad0, magic0);
    }
#define BFLY_MP(RR) \
    case RR: mixed_pass<RR, INV, KIND>(src, dst, n, Ns, magic, twp, t, T, scale, pad0, magic0); break
    switch (R) {
        BFLY_MP(16);
        BFLY_MP(15);
        BFLY_MP(14);
        BFLY_MP(12);
        BFLY_MP(10);
        BFLY_MP(9);
        BFLY_MP(8);
        BFLY_MP(7);
        BFLY_MP(6);
        BFLY_MP(5);
        BFLY_MP(4);
        BFLY_MP(3);
        default: mixed_pass<2, INV, KIND>(src, dst, n, Ns, magic, twp, t, T, scale, pad0, magic0); break;
    }
#undef BFLY_MP
}

template <bool INV, bool WIDE>
__global__ void __launch_bounds__(512, 2) k_mixed(const float2* __restrict__ in, float2* __restrict__ out,
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
        const unsigned mg = a.magic[p];
        const float2* twp = tw + a.twoff[p];
        const bool first = p == 0, last = p == a.passes - 1;
        const float2* s = (p & 1) ? buf0 : buf1;   // written by pass p - 1
        float2* d = (p & 1) ? buf1 : buf0;
        const int p0 = a.pad0;
        const unsigned m0 = a.magic0;
        if (ok) {
            if (first && last) mixed_pass_r<INV, 3, WIDE>(R, src, dst, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (first) mixed_pass_r<INV, 1, WIDE>(R, src, d, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (p == 1 && last) mixed_pass_r<INV, 6, WIDE>(R, s, dst, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (p == 1) mixed_pass_r<INV, 4, WIDE>(R, s, d, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (last) mixed_pass_r<INV, 2, WIDE>(R, s, dst, n, Ns, mg, twp, t, T, scale, p0, m0);
            else mixed_pass_r<INV, 0, WIDE>(R, s, d, n, Ns, mg, twp, t, T, scale, p0, m0);
        }
        if (!last) __syncthreads();
    }
}

// tw[twoff[p] + (r-1) Ns + k] = W_(Ns R)^(k r) = W_n^(k r n / (Ns R)) in FP64, rounded once.
static __global__ void k_tw_mixed(float2* __restrict__ tw, MixedArgs a, int total) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    int p = 1;
    while (p + 1 < a.passes && a.twoff[p + 1] <= i) ++p;
    const int local = i - a.twoff[p], Ns = a.ns[p], R = a.radix[p];
    const int r = local / Ns + 1, k = local % Ns;
    const long long m = (long long)k * r * (a.n / (Ns * R));
    double s, c;
    sincospi(-2.0 * (double)m / (double)a.n, &s, &c);
    tw[i] = make_float2((float)c, (float)s);
}

}  // namespace dev

namespace backend {

namespace {
dev::MixedArgs mixedArgs(const MixedRadix& plan) {
    dev::MixedArgs a{};
    a.n = plan.n;
    a.passes = plan.passes;
    for (int p = 0; p < kMixedMaxPasses; ++p) {
        a.radix[p] = plan.radix[p];
        a.ns[p] = plan.ns[p];
        a.twoff[p] = plan.twoff[p];
        a.magic[p] = plan.ns[p] > 1 ? (unsigned)((0x100000000ull + plan.ns[p] - 1) / (unsigned long long)plan.ns[p]) : 0u;
    }
    return a;
}
bool mixedValid(const MixedRadix& plan) {
    return plan.n >= 2 && (uint32_t)plan.n <= kMixedMaxN && plan.passes >= 1 && plan.passes <= kMixedMaxPasses;
}
}  // namespace

int buildMixedTwiddles(void* tw, const MixedRadix& plan, void* stream) {
    if (!mixedValid(plan)) return (int)cudaErrorInvalidValue;
    if (plan.twsize == 0) return 0;
    dev::k_tw_mixed<<<(plan.twsize + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<float2*>(tw), mixedArgs(plan), plan.twsize);
    return (int)cudaGetLastError();
}

int launchMixed(const void* in, void* out, const MixedRadix& plan, uint64_t batch, bool inverse, float scale,
                const void* tw, void* stream) {
    if (!mixedValid(plan)) return (int)cudaErrorInvalidValue;
    // one butterfly of the largest radix per thread and pass (more of the smaller radices)
    int rmax = 2;
    for (int p = 0; p < plan.passes; ++p) rmax = std::max(rmax, plan.radix[p]);
    // measured on B200 over n = 12..12000: ceil(n / R_max) threads per row with ~200-300 threads
    // per CTA beat n/8 threads per row, larger CTAs, and an 80-register budget
    const int T = std::min(512, (plan.n + rmax - 1) / rmax);
    const int rows = std::max(1, 224 / T);
    constexpr int kMaxSmem = 2 * (dev::spad((int)kMixedMaxN - 1) + 1) * 8;
    static_assert(kMaxSmem <= 227 * 1024, "two rows of the longest length fit in shared memory");
    dev::MixedArgs args = mixedArgs(plan);
    // pass 0 stores at stride R_0: pad its buffer every R_0 slots when R_0 is even (odd strides
    // are conflict-free already), unless that no longer fits; pad 16 is spad's layout
    const int r0 = plan.radix[0];
    int len = dev::spad(plan.n - 1) + 1;
    args.pad0 = (r0 % 2 == 0 && plan.passes > 1) ? r0 : 0;
    if (args.pad0) {
        const int len0 = std::max(len, plan.n + (plan.n - 1) / args.pad0 + 1);
        if (rows * 2 * len0 * 8 <= kMaxSmem) len = len0;
        else args.pad0 = 16;
    }
    args.magic0 = args.pad0 ? (unsigned)((0x100000000ull + args.pad0 - 1) / (unsigned long long)args.pad0) : 0u;
    const int smem = rows * 2 * len * 8;
    bool wide = false;
    for (int p = 0; p < plan.passes; ++p) wide = wide || plan.radix[p] == 11 || plan.radix[p] == 13;
    auto* fn = inverse ? (wide ? dev::k_mixed<true, true> : dev::k_mixed<true, false>)
                       : (wide ? dev::k_mixed<false, true> : dev::k_mixed<false, false>);
    // opted in once per device at kMaxSmem (the largest row pair: n = kMixedMaxN, one row per CTA)
    if (smem > kMaxSmem) return (int)cudaErrorInvalidValue;
    if (int e = optInSharedMemory((const void*)fn, kMaxSmem)) return e;
    const uint64_t grid = (batch + rows - 1) / rows;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, T * rows, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw), args, batch, T,
        rows, len, scale);
    return (int)cudaGetLastError();
}

}  // namespace backend
}  // namespace bfly
