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
#include "istft_ola.cuh"

namespace bfly {
namespace dev {

// ADJ: the adjoint of k_istft (the gradient of an inverse STFT with respect to its spectrum):
// the frames are gathered uncentred from h[p] = g[p - gStart] / envelope(p) (zero outside
// [gStart, gStart + sigLen)), where g is the gradient of the inverse STFT's output, sigLen its
// length and envelope(p) the overlap-added squared window of the frames that exist; the one-sided
// bins are weighted s_edge (k = 0, N/2) and s_int (the rest).
template <int N, int E, int ROWS, bool ADJ>
__global__ void __launch_bounds__((N / 2 / E) * ROWS, min_blocks_64regs((N / 2 / E) * ROWS))
k_stft(const float* __restrict__ sig, float2* __restrict__ out, const float2* __restrict__ tw,
       const float2* __restrict__ twr, const float* __restrict__ window, uint64_t rows,
       uint32_t framesPerSignal, int64_t sigLen, uint64_t sigStride, uint32_t hop, int center, int64_t gStart,
       float s_edge, float s_int) {
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
    // ADJ: 1 / envelope over p mod hop for positions every frame slot of which exists
    // (N - 1 <= p < frames hop); exact sums near either end
    float* rinv = reinterpret_cast<float*>(smem + ROWS * S);
    const int K = (N + (int)hop - 1) / (int)hop;
    if constexpr (ADJ) {
        for (int r = threadIdx.x; r < (int)hop; r += blockDim.x) {
            float e = 0.f;
            for (int j = r; j < N; j += (int)hop) {
                const float w = window ? __ldg(window + j) : 1.f;
                e += w * w;
            }
            rinv[r] = e > 0.f ? 1.f / e : 0.f;
        }
        __syncthreads();
    }
    auto inv = [&](int64_t p) {
        if (p >= N - 1 && p < (int64_t)framesPerSignal * hop) return rinv[p % hop];
        float e = 0.f;
        const int64_t fh = p / hop;
        for (int64_t g = fh - K + 1 > 0 ? fh - K + 1 : 0; g <= fh && g < (int64_t)framesPerSignal; ++g) {
            const int64_t j = p - g * hop;
            if (j < N) {
                const float w = window ? __ldg(window + j) : 1.f;
                e += w * w;
            }
        }
        return e > 0.f ? 1.f / e : 0.f;
    };
    auto sample = [&](int64_t i) {
        if constexpr (ADJ) {
            const int64_t k = i - gStart;
            return k >= 0 && k < sigLen ? __ldg(x + k) * inv(i) : 0.f;
        } else {
            i = i < 0 ? -i : i;
            i = i >= sigLen ? 2 * (sigLen - 1) - i : i;
            return __ldg(x + i);
        }
    };
    // Interior frames starting on an 8-byte boundary (every frame of an even hop away from the
    // padded edges) read one float2 per complex value; the others sample with reflection (ADJ:
    // through the edge envelope and the bounds of g).
    const int64_t at = ADJ ? start - gStart : start;
    const bool direct = ok && at >= 0 && at + N <= sigLen && (reinterpret_cast<uintptr_t>(x + at) & 7u) == 0 &&
                        (!ADJ || (hop % 2 == 0 && start >= N - 1 && start + N <= (int64_t)framesPerSignal * hop));
    const float2* xv = reinterpret_cast<const float2*>(x + (direct ? at : 0));
    float2 v[E];
    TM::run(v, sm, tw, t, rl, [&](int m) {
        if (!ok) return make_float2(0.f, 0.f);
        const int64_t i = start + 2 * m;
        float2 z;
        if (direct) {
            z = __ldg(xv + m);
            if constexpr (ADJ) {   // i even, hop even: i mod hop and i mod hop + 1 are one pair
                const float2 e = *reinterpret_cast<const float2*>(rinv + i % hop);
                z = make_float2(z.x * e.x, z.y * e.y);
            }
        } else {
            z = make_float2(sample(i), sample(i + 1));
        }
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
        const float2 X = cadd(e, cmul<false>(o, wk));
        if constexpr (ADJ) st_stream(dst + k, cscale(X, (k == 0 || k == M) ? s_edge : s_int));
        else st_stream(dst + k, X);
    };
#pragma unroll
    for (int i = 0; i < E; ++i) bin(t + i * T, w[i]);
    if (t == 0) bin(M, wm);
}

// Inverse STFT in one kernel (torch.istft) for power-of-two N: every frame's C2R in registers
// (the k_c2r team), windowed into the row's shared buffer, ROWS frames per wave; the segment
// split, carry, envelope and overlap-add are IstftSegment (istft_ola.cuh).  Frames before the
// CTA's first sample only fill the carry, so K - 1 frames per CTA are transformed twice (Q is
// chosen so that costs < 7%).
// Row stride of the inverse-STFT row buffers: the team's exchange stride rounded up to even.
template <int M, int E>
__host__ __device__ constexpr int istft_row_stride() {
    return smem_stride<M, E, false>() + (smem_stride<M, E, false>() & 1);
}

// ADJ: the adjoint of k_stft (the gradient of an STFT with respect to its signal): bins weighted
// s_edge / s_int (1 and 1/2 for the one-sided transform) instead of irfft's, no envelope, and
// with `pad` = N/2 the reflect padding of a centred STFT folded back (istft_ola.cuh).
template <int N, int E, int ROWS, int MINB, int VEC, bool ADJ>
__global__ void __launch_bounds__((N / 2 / E) * ROWS, MINB)
k_istft(const float2* __restrict__ spec, float* __restrict__ out, const float2* __restrict__ tw,
        const float2* __restrict__ twr, const float* __restrict__ window, uint32_t frames, uint32_t hop, uint32_t Q,
        uint32_t segs, int64_t start, uint64_t outLen, float out_scale, float s_edge, float s_int, int pad) {
    constexpr int M = N / 2;
    constexpr int T = M / E;
    constexpr int CTA = T * ROWS;
    constexpr int S = istft_row_stride<M, E>();   // even: every row buffer 16-byte aligned
    static_assert(2 * S >= N, "a row buffer holds one real frame");
    static_assert(VEC == 1 || VEC == 4, "scalar or float4 overlap-add");
    using TM = Team<M, E, true, sync_kind(T, CTA)>;
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    IstftSegment seg;
    float* scratch = reinterpret_cast<float*>(smem + ROWS * S);
    seg.init(N, hop, frames, Q, segs, start, outLen, window, out, scratch);
    if constexpr (ADJ) seg.initFold(pad, scratch + 2 * (N - (int)hop) + (int)hop);
    const float2* src0 = spec + (uint64_t)(blockIdx.x / segs) * frames * (M + 1);
    float2* sm = smem + rl * S;
    auto row = [&](int r) { return reinterpret_cast<const float*>(smem + r * S); };

    for (uint32_t f0 = seg.fA; f0 < seg.fB; f0 += ROWS) {
        const int R = (int)min((uint32_t)ROWS, seg.fB - f0);
        // rows past R (a CTA's partial first or last wave) transform frame f0 again and are not
        // read: every row runs the same barriers, rows of one warp included
        const float2* src = src0 + (uint64_t)(f0 + (rl < R ? rl : 0)) * (M + 1);
        const float2 nyq = t == 0 ? ld_stream(src + M) : make_float2(0.f, 0.f);
        float2 v[E];
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = ld_stream(src + t + i * T);
        __syncthreads();   // the previous wave is done with the row buffers and the carry
#pragma unroll
        for (int i = 0; i < E; ++i) sm[spad(t + i * T)] = v[i];
        TM::sync(rl);
        TM::load_first(v, t, [&](int k) {
            return c2r_split(sm[spad(k)], k == 0 ? nyq : sm[spad(M - k)], k, __ldg(twr + k), ADJ ? s_edge : 1.f,
                             ADJ ? s_int : 1.f, out_scale);
        });
        TM::sync(rl);
        TM::template passes<0>(v, sm, tw, t, rl);
        TM::sync(rl);
        TM::for_each_out(v, t, [&](int i, float2 z) {   // windowed frame: samples 2i, 2i+1 at sm[i]
            const float2 w = window ? __ldg(reinterpret_cast<const float2*>(window) + i) : make_float2(1.f, 1.f);
            sm[i] = make_float2(z.x * w.x, z.y * w.y);
        });
        __syncthreads();
        seg.template wave<VEC, CTA, ADJ>(f0, R, [&](int r, int j) { return row(r)[j]; },
                                         [&](int r, int j) { return *reinterpret_cast<const float4*>(row(r) + j); });
    }
    seg.zeroTail(segs);
    if constexpr (ADJ) seg.finishFold(segs);
}

}  // namespace dev

namespace backend {

namespace {

// ADJ: the inverse-STFT adjoint (uncentred frames of g / envelope, gStart = the inverse's trim).
template <int N, bool ADJ = false>
int launchStftN(const float* sig, void* out, uint64_t rows, uint32_t framesPerSignal, uint64_t sigLen,
                uint64_t sigStride, uint32_t hop, bool center, const float* window, const void* tw,
                const void* twr, void* stream, int64_t gStart = 0, float sEdge = 1.f, float sInt = 1.f) {
    constexpr int M = N / 2, E = 16, T = M / E;
    constexpr int CTA = T < 256 ? 256 : T;
    constexpr int ROWS = CTA / T;
    constexpr int SMEM = ROWS * dev::smem_stride<M, E, false>() * 8;
    auto* fn = dev::k_stft<N, E, ROWS, ADJ>;
    const int smem = SMEM + (ADJ ? (int)hop * 4 : 0);
    if (int e = optInSharedMemory((const void*)fn, SMEM + (ADJ ? N * 4 : 0))) return e;
    const uint64_t grid = (rows + ROWS - 1) / ROWS;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, CTA, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        sig, static_cast<float2*>(out), static_cast<const float2*>(tw), static_cast<const float2*>(twr), window, rows,
        framesPerSignal, (int64_t)sigLen, sigStride, hop, center ? 1 : 0, gStart, sEdge, sInt);
    return (int)cudaGetLastError();
}

// ADJ: the STFT adjoint (start = pad = N/2 for a centred STFT, else 0), weights 1 / 1/2, scale 1.
template <int N, bool ADJ = false>
int launchIstftN(const float2* spec, float* out, uint64_t signals, uint32_t frames, uint32_t hop, int64_t start,
                 uint64_t outLen, const float* window, const void* tw, const void* twr, float scale, void* stream) {
    constexpr int M = N / 2, E = 16, T = M / E;
    constexpr int CTA = T < 256 ? 256 : T;
    constexpr int ROWS = CTA / T;
    constexpr int ROWBYTES = ROWS * dev::istft_row_stride<M, E>() * 8;
    // N >= 2048: shared memory holds at most 3 CTAs per SM, so up to 80 registers a thread
    constexpr int MINB = N >= 2048 ? 3 : dev::min_blocks_64regs(CTA);
    // float4 overlap-add when the frame starts and the output rows keep 16-byte alignment
    const bool vec = hop % 4 == 0 && outLen % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
    auto* fn = vec ? dev::k_istft<N, E, ROWS, MINB, 4, ADJ> : dev::k_istft<N, E, ROWS, MINB, 1, ADJ>;
    const int pad = ADJ ? (int)start : 0;
    if (int e = optInSharedMemory((const void*)fn, ROWBYTES + 3 * N * 4 + (ADJ ? (N + 2) * 4 : 0))) return e;
    const int smem = ROWBYTES + (2 * (N - (int)hop) + (int)hop) * 4 + (ADJ ? 2 * (pad + 1) * 4 : 0);
    int device = 0, sms = 0, perSm = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, CTA, smem) != cudaSuccess || perSm < 1)
        return (int)cudaErrorInvalidConfiguration;
    uint32_t q, segs;
    istftSegments(N, ROWS, frames, hop, signals, (uint64_t)sms * perSm, &q, &segs);
    if (ADJ && segs > 1) {
        // the first segment must span more than N samples and the last one more than N
        // samples before the end, so each owns both terms of its fold outputs: at least
        // K + 1 frames per segment, a short last segment merged into the one before it
        const uint32_t k1 = (N + hop - 1) / hop + 1;
        if (q < k1) {
            q = k1;
            segs = (frames + q - 1) / q;
        }
        if (segs > 1 && frames - (segs - 1) * q < k1) --segs;
    }
    const uint64_t grid = signals * segs;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, CTA, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        spec, out, static_cast<const float2*>(tw), static_cast<const float2*>(twr), window, frames, hop, q, segs,
        start, outLen, ADJ ? 1.f : scale / N, ADJ ? 1.f : 1.f, ADJ ? 0.5f : 1.f, pad);
    return (int)cudaGetLastError();
}

}  // namespace

int launchIstftAdjoint(const void* gradOut, void* gradSpec, uint32_t n, uint64_t signals, uint32_t frames,
                       uint32_t hop, int64_t start, uint64_t outLen, const void* window, const void* tw,
                       const void* twr, float scale, void* stream) {
    if (!hasStft(n) || hop == 0 || hop > n || frames == 0) return (int)cudaErrorInvalidValue;
    const float* g = static_cast<const float*>(gradOut);
    const float* w = static_cast<const float*>(window);
    const uint64_t rows = signals * frames;
    const float c = scale / (float)n;   // irfft's weights: c at DC and Nyquist, 2c between
#define BFLY_IA(N)                                                                                            \
    case N:                                                                                                   \
        return launchStftN<N, true>(g, gradSpec, rows, frames, outLen, outLen, hop, false, w, tw, twr, stream, \
                                    start, c, 2.f * c)
    switch (n) {
        BFLY_IA(64);
        BFLY_IA(128);
        BFLY_IA(256);
        BFLY_IA(512);
        BFLY_IA(1024);
        BFLY_IA(2048);
        BFLY_IA(4096);
        BFLY_IA(8192);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_IA
}

int launchStftAdjoint(const void* gradSpec, void* gradSig, uint32_t n, uint64_t signals, uint32_t frames,
                      uint32_t hop, bool center, uint64_t sigLen, const void* window, const void* tw, const void* twr,
                      void* stream) {
    if (!hasStft(n) || hop == 0 || hop > n || frames == 0) return (int)cudaErrorInvalidValue;
    if (center && sigLen < (uint64_t)n + 2) return (int)cudaErrorInvalidValue;   // fold regions must not meet
    const float2* x = static_cast<const float2*>(gradSpec);
    float* y = static_cast<float*>(gradSig);
    const float* w = static_cast<const float*>(window);
    const int64_t start = center ? (int64_t)(n / 2) : 0;
#define BFLY_SA(N) \
    case N: return launchIstftN<N, true>(x, y, signals, frames, hop, start, sigLen, w, tw, twr, 1.f, stream)
    switch (n) {
        BFLY_SA(64);
        BFLY_SA(128);
        BFLY_SA(256);
        BFLY_SA(512);
        BFLY_SA(1024);
        BFLY_SA(2048);
        BFLY_SA(4096);
        BFLY_SA(8192);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_SA
}

void istftSegments(uint32_t n, int rows, uint32_t frames, uint32_t hop, uint64_t signals, uint64_t slots,
                   uint32_t* q, uint32_t* segs) {
    // A CTA transforms m*rows frames (m waves), K-1 of them warm-up frames, and stores
    // Q = m*rows - (K-1) frames' worth of samples.  Estimated time = rounds of resident CTAs x
    // waves per CTA; the smallest wins, ties going to the larger m (fewer warm-up frames).
    const uint32_t k1 = (n + hop - 1) / hop - 1;
    const uint64_t r = (uint64_t)rows;
    const uint64_t mlo = (k1 + 1 + r - 1) / r;
    const uint64_t mhi = (17ull * k1 + (k1 ? 0 : 16) + r - 1) / r + 64;
    uint64_t best = ~0ull;
    *q = (uint32_t)(mlo * r - k1);
    *segs = (uint32_t)((frames + *q - 1) / *q);
    for (uint64_t m = mlo; m <= mhi; ++m) {
        const uint64_t qq = m * r - k1;
        const uint64_t sg = (frames + qq - 1) / qq;
        const uint64_t rounds = (signals * sg + slots - 1) / (slots ? slots : 1);
        if (rounds * m <= best) {
            best = rounds * m;
            *q = (uint32_t)qq;
            *segs = (uint32_t)sg;
        }
        if (sg == 1) break;
    }
}

bool hasStft(uint32_t n) { return n >= kStftMinN && n <= kStftMaxN && !(n & (n - 1)); }

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

int launchIstft(const void* spec, void* out, uint32_t n, uint64_t signals, uint32_t frames, uint32_t hop,
                int64_t start, uint64_t outLen, const void* window, const void* tw, const void* twr, float scale,
                void* stream) {
    if (!hasStft(n) || hop == 0 || hop > n || frames == 0) return (int)cudaErrorInvalidValue;
    const float2* x = static_cast<const float2*>(spec);
    float* y = static_cast<float*>(out);
    const float* w = static_cast<const float*>(window);
#define BFLY_IS(N) \
    case N: return launchIstftN<N>(x, y, signals, frames, hop, start, outLen, w, tw, twr, scale, stream)
    switch (n) {
        BFLY_IS(64);
        BFLY_IS(128);
        BFLY_IS(256);
        BFLY_IS(512);
        BFLY_IS(1024);
        BFLY_IS(2048);
        BFLY_IS(4096);
        BFLY_IS(8192);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_IS
}

}  // namespace backend
}  // namespace bfly
