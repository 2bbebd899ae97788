// C2C of any length n in [2, 8192] (used for the non-power-of-two ones) by Bluestein's chirp-z
// algorithm, one CTA team per row, one HBM pass:
//   X[k] = c[k] * sum_j (x[j] c[j]) * conj(c[k-j]),   c[m] = exp(-i*pi*m^2/n)   (forward)
// (from jk = (j^2 + k^2 - (k-j)^2)/2).  The sum is a linear convolution, computed as a cyclic
// one of length M = max(64, next power of two >= 2n-1):
//   a[j] = x[j] c[j] (j < n, else 0);  h[m] = conj(c[m]) for m < n, h[M-m] = conj(c[m]) for
//   0 < m < n, else 0;  conv = IFFT_M(FFT_M(a) * FFT_M(h)).
// FFT_M(h) / M (the filter) and c are built per (plan, n) in FP64 on the device and rounded
// to fp32.  The kernel loads x*c zero-padded, runs the forward M-point Stockham FFT in
// registers and shared memory, multiplies by the filter, re-enters the inverse FFT through
// shared memory, multiplies by c and stores the first n outputs.  The inverse transform uses
// conj(c) and conj(filter): h is symmetric (h[M-m] = h[m]), so the filter of conj(h) is the
// conjugate of the filter of h.
#include <cuda_runtime.h>

#include "backend.h"
#include "fft_kernels.cuh"

namespace bfly {
namespace dev {

// `x`, as an opaque value that is only available once `dep` has been computed.
__device__ __forceinline__ int opaque(int x, float dep) {
    int r;
    asm volatile("mov.b32 %0, %1;" : "=r"(r) : "r"(x), "f"(dep));
    return r;
}

template <int M, int E, int ROWS, bool INV>
__global__ void __launch_bounds__((M / E) * ROWS, min_blocks_64regs((M / E) * ROWS))
k_bluestein(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
            const float2* __restrict__ chirp, const float2* __restrict__ filt, uint32_t n, uint64_t batch,
            float scale) {
    constexpr int T = M / E;
    constexpr int S = smem_stride<M, E, false>();
    constexpr int SYNC = sync_kind(T, T * ROWS);
    using TF = Team<M, E, false, SYNC>;
    using TI = Team<M, E, true, SYNC>;
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * ROWS + rl;
    const bool ok = row < batch;
    const float2* src = in + row * n;
    float2* dst = out + row * n;
    float2* sm = smem + rl * S;
    const int len = (int)n;
    float2 v[E];
    TF::run(v, sm, tw, t, rl, [&](int i) {
        return (ok && i < len) ? cmul<INV>(ld_stream(src + i), __ldg(chirp + i)) : make_float2(0.f, 0.f);
    });
    TF::for_each_slot(v, t, [&](int k, float2& x) { x = cmul<INV>(x, __ldg(filt + k)); });
    TF::sync(rl);   // the last forward pass has read the exchange buffer
    TF::for_each_out(v, t, [&](int k, float2 x) { sm[spad(k)] = x; });
    TF::sync(rl);
    // Both transforms derive the same shared-memory and twiddle addresses from t; left alone the
    // compiler computes them once and keeps them all live through both halves (over 160
    // registers).  The inverse half takes opaque copies of t and of the buffer, recomputed here.
    const int ti = opaque(t, v[0].x);
    float2* smi = smem + opaque(rl, v[0].x) * S;
    TI::load_first(v, ti, [&](int i) { return smi[spad(i)]; });
    TI::sync(rl);   // the inverse passes reuse the buffer
    TI::template passes<0>(v, smi, tw, ti, rl);
    if (ok)
        TI::for_each_out(v, ti, [&](int k, float2 x) {
            if (k < len) st_stream(dst + k, cscale(cmul<INV>(x, __ldg(chirp + k)), scale));
        });
}

// c[j] = exp(-i*pi*(j^2 mod 2n)/n) for j < n (fp32), and the zero-padded symmetric sequence
// h (FP64, M entries) whose transform is the filter.
static __global__ void k_bluestein_chirp(float2* __restrict__ chirp, double2* __restrict__ h, uint32_t n,
                                         uint32_t M) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const uint32_t j = m < n ? m : (M - m < n ? M - m : 0u);
    const bool live = m < n || M - m < n;
    double s = 0.0, c = 0.0;
    if (live) {
        const uint64_t q = ((uint64_t)j * j) % (2ull * n);
        sincospi(-(double)q / (double)n, &s, &c);
    }
    h[m] = live ? make_double2(c, -s) : make_double2(0.0, 0.0);   // conj(c[j])
    if (m < n) chirp[m] = make_float2((float)c, (float)s);
}

// filt[k] = (1/M) * sum_m h[m] exp(-2*pi*i*m*k/M), direct sum in FP64 over the 2n-1 nonzero m.
static __global__ void k_bluestein_filter(float2* __restrict__ filt, const double2* __restrict__ h, uint32_t n,
                                          uint32_t M) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    double re = 0.0, im = 0.0;
    auto term = [&](uint32_t m) {
        const uint64_t q = ((uint64_t)m * k) % M;
        double s, c;
        sincospi(-2.0 * (double)q / (double)M, &s, &c);
        const double2 a = h[m];
        re += a.x * c - a.y * s;
        im += a.x * s + a.y * c;
    };
    for (uint32_t m = 0; m < n; ++m) term(m);
    for (uint32_t m = M - n + 1; m < M; ++m) term(m);
    filt[k] = make_float2((float)(re / M), (float)(im / M));
}

}  // namespace dev

namespace backend {

namespace {

template <int M, bool INV>
int launchBluesteinM(const void* in, void* out, uint32_t n, uint64_t batch, float scale, const void* tw,
                     const void* chirp, const void* filt, void* stream) {
    constexpr int E = 16, T = M / E;
    constexpr int CTA = T < 256 ? 256 : T;
    constexpr int ROWS = CTA / T;
    constexpr int SMEM = ROWS * dev::smem_stride<M, E, false>() * 8;
    auto* fn = dev::k_bluestein<M, E, ROWS, INV>;
    if (int e = optInSharedMemory((const void*)fn, SMEM)) return e;
    const uint64_t grid = (batch + ROWS - 1) / ROWS;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, CTA, SMEM, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(tw),
        static_cast<const float2*>(chirp), static_cast<const float2*>(filt), n, batch, scale);
    return (int)cudaGetLastError();
}

}  // namespace

uint32_t bluesteinM(uint32_t n) {
    if (n < 2 || n > kBluesteinMaxN) return 0;
    uint32_t m = 64;
    while (m < 2 * n - 1) m <<= 1;
    return m;
}

int buildBluesteinTables(void* chirp, void* filt, void* scratch, uint32_t n, void* stream) {
    const uint32_t M = bluesteinM(n);
    if (!M) return (int)cudaErrorInvalidValue;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned blocks = (M + 255) / 256;
    dev::k_bluestein_chirp<<<blocks, 256, 0, s>>>(static_cast<float2*>(chirp), static_cast<double2*>(scratch), n, M);
    dev::k_bluestein_filter<<<blocks, 256, 0, s>>>(static_cast<float2*>(filt), static_cast<const double2*>(scratch),
                                                   n, M);
    return (int)cudaGetLastError();
}

int launchBluestein(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale,
                    const void* tw, const void* chirp, const void* filt, void* stream) {
#define BFLY_BS(M)                                                                             \
    case M:                                                                                    \
        return inverse ? launchBluesteinM<M, true>(in, out, n, batch, scale, tw, chirp, filt, stream) \
                       : launchBluesteinM<M, false>(in, out, n, batch, scale, tw, chirp, filt, stream)
    switch (bluesteinM(n)) {
        BFLY_BS(64);
        BFLY_BS(128);
        BFLY_BS(256);
        BFLY_BS(512);
        BFLY_BS(1024);
        BFLY_BS(2048);
        BFLY_BS(4096);
        BFLY_BS(8192);
        BFLY_BS(16384);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_BS
}

}  // namespace backend
}  // namespace bfly
