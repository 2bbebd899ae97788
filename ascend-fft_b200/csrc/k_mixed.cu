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
// argument, so one kernel (per radix class) serves every such length; the plans of common
// lengths also have kernels with the pass list fixed at compile time (FixedRows), whose
// constant offsets and strides fold into the loads and stores (37 % fewer instructions at
// n = 1000).
// This unit: the twiddle kernel and the launchers; the kernels are in mixed.cuh.
#include "mixed.cuh"

namespace bfly {
namespace dev {

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

namespace {
// Launch shape of the mixed-radix kernels for one M-point complex row (k_mixed and the real
// transforms built on it): threads per row, rows per CTA, buffer length and the pass-0 pad.
struct MixedShape {
    dev::MixedArgs args;
    int T = 0, rows = 0, len = 0, smem = 0;
    int cls = 0;   // radix class of the kernel instance (mixed_pass_r)
};
constexpr int kMixedMaxSmem = 227 * 1024;
static_assert(2 * (dev::spad((int)kMixedMaxN - 1) + 1) * 8 <= kMixedMaxSmem, "two rows of the longest length fit in shared memory");

MixedShape mixedShape(const MixedRadix& plan) {
    MixedShape m;
    m.args = mixedArgs(plan);
    // one butterfly of the largest radix per thread and pass (more of the smaller radices);
    // measured on B200 over n = 12..12000: ceil(n / R_max) threads per row with ~200-300
    // threads per CTA beat n/8 threads per row, larger CTAs, and an 80-register budget
    int rmax = 2;
    for (int p = 0; p < plan.passes; ++p) {
        rmax = std::max(rmax, plan.radix[p]);
        m.cls = std::max(m.cls, plan.radix[p] == 11 || plan.radix[p] == 13 ? 2 : plan.radix[p] > 10 ? 1 : 0);
    }
    m.T = std::min(512, (plan.n + rmax - 1) / rmax);
    m.rows = std::max(1, 224 / m.T);
    // pass 0 stores at stride R_0: pad its buffer every R_0 slots when R_0 is even (odd strides
    // are conflict-free already), unless that no longer fits (then it stays unpadded)
    const int r0 = plan.radix[0];
    m.len = dev::spad(plan.n - 1) + 1;
    m.args.pad0 = (r0 % 2 == 0 && plan.passes > 1) ? r0 : 0;
    if (m.args.pad0) {
        const int len0 = std::max(m.len, plan.n + (plan.n - 1) / m.args.pad0 + 1);
        if (m.rows * 2 * len0 * 8 <= kMixedMaxSmem) m.len = len0;
        else m.args.pad0 = 0;
    }
    m.args.magic0 =
        m.args.pad0 ? (unsigned)((0x100000000ull + m.args.pad0 - 1) / (unsigned long long)m.args.pad0) : 0u;
    m.smem = m.rows * 2 * m.len * 8;
    return m;
}

MixedKernels kernelsFor(const MixedRadix& plan, const MixedShape& m) {
    int count = 0;
    const FixedEntry* fixed = mixedFixed(&count);
    for (int i = 0; i < count; ++i) {
        const FixedEntry& e = fixed[i];
        if (e.passes != plan.passes || e.T != m.T || e.pad0 != m.args.pad0) continue;
        bool same = true;
        for (int p = 0; p < e.passes; ++p) same = same && e.radix[p] == plan.radix[p];
        if (same) return e.k;
    }
    static const MixedKernels generic[3] = {mixedGeneric0(), mixedGeneric1(), mixedGeneric2()};
    return generic[m.cls];
}
}  // namespace

int launchMixed(const void* in, void* out, const MixedRadix& plan, uint64_t batch, bool inverse, float scale,
                const void* tw, void* stream) {
    if (!mixedValid(plan)) return (int)cudaErrorInvalidValue;
    const MixedShape m = mixedShape(plan);
    const MixedKernels k = kernelsFor(plan, m);
    auto* fn = inverse ? k.inv : k.fwd;
    // opted in once per device at kMixedMaxSmem
    if (m.smem > kMixedMaxSmem) return (int)cudaErrorInvalidValue;
    if (int e = optInSharedMemory((const void*)fn, kMixedMaxSmem)) return e;
    const uint64_t groups = (batch + m.rows - 1) / m.rows;
    if (groups > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)groups, m.T * m.rows, m.smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw), m.args, batch, m.T,
        m.rows, m.len, scale);
    return (int)cudaGetLastError();
}

int launchR2CMixed(const void* in, void* out, const MixedRadix& half, uint64_t batch, const void* tw, const void* twr,
                   float sEdge, float sInt, void* stream) {
    if (!mixedValid(half)) return (int)cudaErrorInvalidValue;
    const MixedShape m = mixedShape(half);
    auto* fn = kernelsFor(half, m).r2c;
    if (m.smem > kMixedMaxSmem) return (int)cudaErrorInvalidValue;
    if (int e = optInSharedMemory((const void*)fn, kMixedMaxSmem)) return e;
    const uint64_t groups = (batch + m.rows - 1) / m.rows;
    if (groups > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)groups, m.T * m.rows, m.smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw),
        static_cast<const float2*>(twr), m.args, batch, m.T, m.rows, m.len, sEdge, sInt);
    return (int)cudaGetLastError();
}

int launchC2RMixed(const void* in, void* out, const MixedRadix& half, uint64_t batch, const void* tw, const void* twr,
                   float sEdge, float sInt, float outScale, void* stream) {
    if (!mixedValid(half)) return (int)cudaErrorInvalidValue;
    const MixedShape m = mixedShape(half);
    auto* fn = kernelsFor(half, m).c2r;
    if (m.smem > kMixedMaxSmem) return (int)cudaErrorInvalidValue;
    if (int e = optInSharedMemory((const void*)fn, kMixedMaxSmem)) return e;
    const uint64_t groups = (batch + m.rows - 1) / m.rows;
    if (groups > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)groups, m.T * m.rows, m.smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw),
        static_cast<const float2*>(twr), m.args, batch, m.T, m.rows, m.len, sEdge, sInt, outScale);
    return (int)cudaGetLastError();
}

int launchStftMixed(const void* sig, void* out, const MixedRadix& half, uint64_t signals, uint32_t framesPerSignal,
                    uint64_t sigLen, uint64_t sigStride, uint32_t hop, bool center, const void* window,
                    const void* tw, const void* twr, void* stream) {
    if (!mixedValid(half)) return (int)cudaErrorInvalidValue;
    const MixedShape m = mixedShape(half);
    auto* fn = kernelsFor(half, m).stft;
    if (m.smem > kMixedMaxSmem) return (int)cudaErrorInvalidValue;
    if (int e = optInSharedMemory((const void*)fn, kMixedMaxSmem)) return e;
    const uint64_t frames = signals * framesPerSignal;
    const uint64_t groups = (frames + m.rows - 1) / m.rows;
    if (groups > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)groups, m.T * m.rows, m.smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float*>(sig), static_cast<float2*>(out), static_cast<const float2*>(tw),
        static_cast<const float2*>(twr), static_cast<const float*>(window), m.args, frames, framesPerSignal,
        (int64_t)sigLen, sigStride, hop, center ? 1 : 0, m.T, m.rows, m.len);
    return (int)cudaGetLastError();
}

int launchIstftMixed(const void* spec, void* out, const MixedRadix& half, uint64_t signals, uint32_t frames,
                     uint32_t hop, int64_t start, uint64_t outLen, const void* window, const void* tw, const void* twr,
                     float scale, void* stream) {
    if (!mixedValid(half)) return (int)cudaErrorInvalidValue;
    const int N = 2 * half.n;
    if (N > (int)kIstftMixedMaxN || hop == 0 || hop > (uint32_t)N || frames == 0) return (int)cudaErrorInvalidValue;
    MixedShape m = mixedShape(half);
    m.len += m.len & 1;   // even: every row buffer 16-byte aligned for the float4 overlap-add
    const int smem = m.rows * 2 * m.len * 8 + (2 * (N - (int)hop) + (int)hop) * 4;
    // opted in once per kernel at the largest case: rows * 2 * len of the longest plan plus
    // carry and envelope of N = kIstftMixedMaxN
    constexpr int kMaxSmem = 227 * 1024;
    if (smem > kMaxSmem) return (int)cudaErrorInvalidValue;
    // float4 overlap-add: frame, hop and output lengths multiples of 4, 16-byte aligned output
    // and window (a frame of N % 4 == 2 would read past its row)
    const bool vec = N % 4 == 0 && hop % 4 == 0 && outLen % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0 &&
                     (reinterpret_cast<uintptr_t>(window) & 15u) == 0;
    const MixedKernels k = kernelsFor(half, m);
    auto* fn = vec ? k.istft4 : k.istft1;
    if (int e = optInSharedMemory((const void*)fn, kMaxSmem)) return e;
    int device = 0, sms = 0, perSm = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, m.T * m.rows, smem) != cudaSuccess || perSm < 1)
        return (int)cudaErrorInvalidConfiguration;
    uint32_t q, segs;
    istftSegments((uint32_t)N, m.rows, frames, hop, signals, (uint64_t)sms * perSm, &q, &segs);
    const uint64_t grid = signals * segs;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, m.T * m.rows, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(spec), static_cast<float*>(out), static_cast<const float2*>(tw),
        static_cast<const float2*>(twr), static_cast<const float*>(window), m.args, frames, hop, q, segs, start,
        outLen, scale / N, m.T, m.rows, m.len);
    return (int)cudaGetLastError();
}

}  // namespace backend
}  // namespace bfly
