// Short-time Fourier transform in one kernel: frame gather (hop, optional centred reflect
// padding) x window, N/2-point complex FFT of the packed frame and the R2C split epilogue.
//   frame f of signal s:  y[j] = w[j] * x_s[f*hop + j - (center ? N/2 : 0)],  j < N,
//   positions outside [0, L) reflected (x[-i] = x[i], x[L-1+i] = x[L-1-i]) as torch.stft's
//   default pad_mode="reflect";  out[s][f][k] = sum_j y[j] exp(-2*pi*i*j*k/N), k <= N/2.
// Frames overlap, so samples are read through the read-only cache (L1/L2 reuse across the
// N/hop frames that cover them) instead of the streaming path of the batched transforms.
// The reference runs its STFT cases as a dense-frame R2C proxy (docs/testing.md:118,
// config/test_matrix.json "stft": R2C with batch = frames); framing, windowing and overlap
// are done here inside the transform.
#include <cuda_runtime.h>

#include "backend.h"
#include "fft_kernels.cuh"

namespace bfly {
namespace dev {

template <int N, int E, int ROWS>
__global__ void __launch_bounds__((N / 2 / E) * ROWS, min_blocks_64regs((N / 2 / E) * ROWS))
k_stft(const float* __restrict__ sig, float2* __restrict__ out, const float2* __restrict__ tw,
       const float2* __restrict__ twr, const float* __restrict__ window, uint64_t rows,
       uint32_t framesPerSignal, int64_t sigLen, uint64_t sigStride, uint32_t hop, int center) {
    constexpr int M = N / 2;
    constexpr int T = M / E;
    constexpr int S = smem_stride<M, E, false>();
    using TM = Team<M, E, false, sync_kind(T, T * ROWS)>;
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * ROWS + rl;
    const bool ok = row < rows;
    const uint64_t s = ok ? row / framesPerSignal : 0;
    const uint64_t f = ok ? row % framesPerSignal : 0;
    const float* x = sig + s * sigStride;
    const int64_t start = (int64_t)f * hop - (center ? N / 2 : 0);
    float2* dst = out + row * (M + 1);
    float2* sm = smem + rl * S;
    auto sample = [&](int64_t i) {
        i = i < 0 ? -i : i;
        i = i >= sigLen ? 2 * (sigLen - 1) - i : i;
        return __ldg(x + i);
    };
    // Interior frames starting on an 8-byte boundary (every frame of an even hop away from the
    // padded edges) read one float2 per complex value; the others sample with reflection.
    const bool direct = ok && start >= 0 && start + N <= sigLen &&
                        (reinterpret_cast<uintptr_t>(x + start) & 7u) == 0;
    const float2* xv = reinterpret_cast<const float2*>(x + (direct ? start : 0));
    float2 v[E];
    TM::run(v, sm, tw, t, rl, [&](int m) {
        if (!ok) return make_float2(0.f, 0.f);
        const int64_t i = start + 2 * m;
        float2 z = direct ? __ldg(xv + m) : make_float2(sample(i), sample(i + 1));
        if (window) {
            const float2 w = __ldg(reinterpret_cast<const float2*>(window) + m);
            z = make_float2(z.x * w.x, z.y * w.y);
        }
        return z;
    });
    float2 w[E];
#pragma unroll
    for (int i = 0; i < E; ++i) w[i] = __ldg(twr + t + i * T);
    const float2 wm = __ldg(twr + M);
    TM::sync(rl);
    TM::for_each_out(v, t, [&](int i, float2 z) { sm[spad(i)] = z; });
    TM::sync(rl);
    if (!ok) return;
    auto bin = [&](int k, float2 wk) {
        const float2 a = sm[spad(k & (M - 1))];
        const float2 b = sm[spad((M - k) & (M - 1))];
        const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
        const float2 o = make_float2(0.5f * (a.y + b.y), 0.5f * (b.x - a.x));
        st_stream(dst + k, cadd(e, cmul<false>(o, wk)));
    };
#pragma unroll
    for (int i = 0; i < E; ++i) bin(t + i * T, w[i]);
    if (t == 0) bin(M, wm);
}

// Overlap-add of inverse-transformed frames (the second half of an inverse STFT), gather form:
//   out[s][i] = sum_f w[j] fr[s][f][j] / sum_f w[j]^2,   j = i + start - f*hop, 0 <= j < n,
// with w = 1 when window is null; start = n/2 removes the centring pad.  One thread per output
// sample; the frames covering it are read at consecutive j by consecutive threads.  Samples
// whose envelope is zero are written as 0 (the caller checks the envelope beforehand).
static __global__ void k_ola(const float* __restrict__ fr, float* __restrict__ out, const float* __restrict__ window,
                             uint32_t n, uint32_t frames, uint32_t hop, int64_t start, uint64_t outLen,
                             uint64_t signals) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= outLen * signals) return;
    const uint64_t s = g / outLen, i = g % outLen;
    const int64_t p = (int64_t)i + start;   // position in the padded signal
    const float* f0 = fr + s * (uint64_t)frames * n;
    int64_t fhi = p / hop;
    if (fhi > (int64_t)frames - 1) fhi = (int64_t)frames - 1;
    int64_t flo = p - (int64_t)n + 1 > 0 ? (p - (int64_t)n + hop) / hop : 0;
    float acc = 0.f, env = 0.f;
    for (int64_t f = flo; f <= fhi; ++f) {
        const int64_t j = p - f * (int64_t)hop;
        if (j < 0 || j >= (int64_t)n) continue;
        const float w = window ? __ldg(window + j) : 1.f;
        acc += w * __ldg(f0 + (uint64_t)f * n + j);
        env += w * w;
    }
    out[g] = env > 0.f ? acc / env : 0.f;
}

}  // namespace dev

namespace backend {

namespace {

template <int N>
int launchStftN(const float* sig, void* out, uint64_t rows, uint32_t framesPerSignal, uint64_t sigLen,
                uint64_t sigStride, uint32_t hop, bool center, const float* window, const void* tw,
                const void* twr, void* stream) {
    constexpr int M = N / 2, E = 16, T = M / E;
    constexpr int CTA = T < 256 ? 256 : T;
    constexpr int ROWS = CTA / T;
    constexpr int SMEM = ROWS * dev::smem_stride<M, E, false>() * 8;
    auto* fn = dev::k_stft<N, E, ROWS>;
    if (int e = optInSharedMemory((const void*)fn, SMEM)) return e;
    const uint64_t grid = (rows + ROWS - 1) / ROWS;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, CTA, SMEM, reinterpret_cast<cudaStream_t>(stream)>>>(
        sig, static_cast<float2*>(out), static_cast<const float2*>(tw), static_cast<const float2*>(twr), window, rows,
        framesPerSignal, (int64_t)sigLen, sigStride, hop, center ? 1 : 0);
    return (int)cudaGetLastError();
}

}  // namespace

bool hasStft(uint32_t n) { return n >= kStftMinN && n <= kStftMaxN && !(n & (n - 1)); }

int launchOla(const void* frames, void* out, uint32_t n, uint64_t signals, uint32_t framesPerSignal, uint32_t hop,
              int64_t start, uint64_t outLen, const void* window, void* stream) {
    const uint64_t total = outLen * signals;
    if (total == 0) return 0;
    const uint64_t blocks = (total + 255) / 256;
    if (blocks > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    dev::k_ola<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float*>(frames), static_cast<float*>(out), static_cast<const float*>(window), n,
        framesPerSignal, hop, start, outLen, signals);
    return (int)cudaGetLastError();
}

int launchStft(const void* sig, void* out, uint32_t n, uint64_t signals, uint32_t framesPerSignal,
               uint64_t sigLen, uint64_t sigStride, uint32_t hop, bool center, const void* window,
               const void* tw, const void* twr, void* stream) {
    const float* x = static_cast<const float*>(sig);
    const float* w = static_cast<const float*>(window);
    const uint64_t rows = signals * framesPerSignal;
#define BFLY_ST(N) \
    case N: return launchStftN<N>(x, out, rows, framesPerSignal, sigLen, sigStride, hop, center, w, tw, twr, stream)
    switch (n) {
        BFLY_ST(64);
        BFLY_ST(128);
        BFLY_ST(256);
        BFLY_ST(512);
        BFLY_ST(1024);
        BFLY_ST(2048);
        BFLY_ST(4096);
        BFLY_ST(8192);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_ST
}

}  // namespace backend
}  // namespace bfly
