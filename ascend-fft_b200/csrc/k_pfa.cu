// C2C of n = A*B (A in {3, 5, 9, 15}, B a power of two >= 16, n <= 12288) by the Good-Thomas
// prime-factor mapping, one HBM pass.  With gcd(A, B) = 1,
//   input  j <-> (j1, j2) = (j mod A, j mod B)          (Chinese-remainder map)
//   output k  =  (B*k1 + A*k2) mod n                     (Ruritanian map)
// gives W_n^(j*k) = W_A^(j1*k1) * W_B^(j2*k2), so the n-point DFT is an A x B two-dimensional
// DFT with no twiddle factors between the dimensions:
//   X[(B k1 + A k2) mod n] = sum_j1 W_A^(j1 k1) sum_j2 W_B^(j2 k2) x[j with j mod A = j1, j mod B = j2].
// One team of n/16 threads per row: coalesced loads scattered into a shared [A][B] array,
// A sub-teams run the B-point Stockham FFT (Team), direct A-point DFTs down the B columns
// write the outputs at their natural positions, then coalesced stores.
#include <cuda_runtime.h>

#include "backend.h"
#include "fft_kernels.cuh"

namespace bfly {
namespace dev {

template <int A, int B>
struct Pfa {
    static constexpr int N = A * B, E = 16;
    static constexpr int TR = B / E;                      // threads per B-point sub-row
    static constexpr int T = A * TR;                      // threads per n-point row
    static constexpr int SB = smem_stride<B, E, false>(); // sub-row stride (padded exchange)
    static constexpr int NAT = spad(N - 1) + 1;           // natural-order staging extent
    static constexpr int ROWBUF = (A * SB > NAT ? A * SB : NAT) | 1;
    static constexpr int CTA = T < 256 ? (256 / T) * T : T;
    static constexpr int ROWS = CTA / T;
    static constexpr int COLS = (B + T - 1) / T;          // columns of the A-point phase per thread
    // n <= 12288: the A = 15, n = 15360 variant would need 960 threads and spills its columns
    static_assert(A % 2 == 1 && B % E == 0 && N <= (int)backend::kPfaMaxN, "shape outside the instantiated family");
};

template <int A, int B, bool INV>
__global__ void __launch_bounds__(Pfa<A, B>::CTA)
k_pfa(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ twB,
      const float2* __restrict__ wA, uint64_t batch, float scale) {
    using P = Pfa<A, B>;
    constexpr int E = P::E, N = P::N, T = P::T;
    using TB = Team<B, E, INV, kSyncBlock>;   // every sync below is block-wide: all rows of the
                                             // CTA run the same number of barriers
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int tid = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * P::ROWS + rl;
    const bool ok = row < batch;
    const float2* src = in + row * N;
    float2* dst = out + row * N;
    float2* buf = smem + rl * P::ROWBUF;

    // 1. coalesced loads, scattered to [j mod A][j mod B]
#pragma unroll 4
    for (int i = 0; i < E; ++i) {
        const int j = tid + i * T;
        buf[(j % A) * P::SB + spad(j % B)] = ok ? ld_stream(src + j) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    // 2. B-point FFT of sub-row j1 by sub-team j1, results back in natural order k2
    {
        const int j1 = tid / P::TR, t = tid % P::TR;
        float2* sub = buf + j1 * P::SB;
        float2 v[E];
        TB::load_first(v, t, [&](int i) { return sub[spad(i)]; });
        __syncthreads();
        TB::template passes<0>(v, sub, twB, t, 0);
        __syncthreads();
        TB::for_each_out(v, t, [&](int k2, float2 x) { sub[spad(k2)] = x; });
    }
    __syncthreads();
    // 3. A-point DFT down each column k2; outputs to X[(B k1 + A k2) mod n] in natural order
    float2 w[A];
#pragma unroll
    for (int m = 0; m < A; ++m) w[m] = __ldg(wA + m);
    float2 col[P::COLS][A];
#pragma unroll
    for (int c = 0; c < P::COLS; ++c) {
        const int k2 = tid + c * T;
#pragma unroll
        for (int j1 = 0; j1 < A; ++j1) col[c][j1] = k2 < B ? buf[j1 * P::SB + spad(k2)] : make_float2(0.f, 0.f);
    }
    __syncthreads();   // every column is in registers: the buffer is free for natural order
#pragma unroll
    for (int c = 0; c < P::COLS; ++c) {
        const int k2 = tid + c * T;
        if (k2 < B) {
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) {
                float2 acc = col[c][0];
#pragma unroll
                for (int j1 = 1; j1 < A; ++j1) acc = cadd(acc, cmul<INV>(col[c][j1], w[(j1 * k1) % A]));
                buf[spad((B * k1 + A * k2) % N)] = acc;
            }
        }
    }
    __syncthreads();
    // 4. coalesced stores
    if (ok) {
#pragma unroll 4
        for (int i = 0; i < E; ++i) {
            const int k = tid + i * T;
            st_stream(dst + k, cscale(buf[spad(k)], scale));
        }
    }
}

}  // namespace dev

namespace backend {

namespace {

template <int A, int B, bool INV>
int launchPfaAB(const void* in, void* out, uint64_t batch, float scale, const void* twB, const void* wA,
                void* stream) {
    using P = dev::Pfa<A, B>;
    constexpr int SMEM = P::ROWS * P::ROWBUF * 8;
    auto* fn = dev::k_pfa<A, B, INV>;
    if (int e = optInSharedMemory((const void*)fn, SMEM)) return e;
    const uint64_t grid = (batch + P::ROWS - 1) / P::ROWS;
    if (grid > 0x7fffffffull) return (int)cudaErrorInvalidValue;
    fn<<<(unsigned)grid, P::CTA, SMEM, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const float2*>(twB),
        static_cast<const float2*>(wA), batch, scale);
    return (int)cudaGetLastError();
}

template <int A, bool INV>
int launchPfaA(const void* in, void* out, uint32_t b, uint64_t batch, float scale, const void* twB,
               const void* wA, void* stream) {
    switch (b) {
        case 16: return launchPfaAB<A, 16, INV>(in, out, batch, scale, twB, wA, stream);
        case 32: return launchPfaAB<A, 32, INV>(in, out, batch, scale, twB, wA, stream);
        case 64: return launchPfaAB<A, 64, INV>(in, out, batch, scale, twB, wA, stream);
        case 128: return launchPfaAB<A, 128, INV>(in, out, batch, scale, twB, wA, stream);
        case 256: return launchPfaAB<A, 256, INV>(in, out, batch, scale, twB, wA, stream);
        case 512: return launchPfaAB<A, 512, INV>(in, out, batch, scale, twB, wA, stream);
        case 1024:
            if constexpr (A * 1024 <= kPfaMaxN) return launchPfaAB<A, 1024, INV>(in, out, batch, scale, twB, wA, stream);
            break;
        case 2048:
            if constexpr (A * 2048 <= kPfaMaxN) return launchPfaAB<A, 2048, INV>(in, out, batch, scale, twB, wA, stream);
            break;
        case 4096:
            if constexpr (A * 4096 <= kPfaMaxN) return launchPfaAB<A, 4096, INV>(in, out, batch, scale, twB, wA, stream);
            break;
        default: break;
    }
    return (int)cudaErrorInvalidValue;
}

}  // namespace

bool pfaSplit(uint32_t n, uint32_t* a, uint32_t* b) {
    *a = *b = 0;
    for (uint32_t A : {3u, 5u, 9u, 15u}) {
        if (n % A) continue;
        const uint32_t B = n / A;
        if (B >= 16 && !(B & (B - 1)) && n <= kPfaMaxN) {
            *a = A;
            *b = B;
        }
    }
    return *a != 0;
}

int launchPfa(const void* in, void* out, uint32_t n, uint64_t batch, bool inverse, float scale, const void* twB,
              const void* wA, void* stream) {
    uint32_t a = 0, b = 0;
    if (!pfaSplit(n, &a, &b)) return (int)cudaErrorInvalidValue;
#define BFLY_PFA(A) \
    return inverse ? launchPfaA<A, true>(in, out, b, batch, scale, twB, wA, stream) \
                   : launchPfaA<A, false>(in, out, b, batch, scale, twB, wA, stream)
    switch (a) {
        case 3: BFLY_PFA(3);
        case 5: BFLY_PFA(5);
        case 9: BFLY_PFA(9);
        case 15: BFLY_PFA(15);
        default: return (int)cudaErrorInvalidValue;
    }
#undef BFLY_PFA
}

}  // namespace backend
}  // namespace bfly
