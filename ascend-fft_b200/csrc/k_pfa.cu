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
#include "fft_odd.cuh"

namespace bfly {
namespace dev {

// In-place A-point DFT of x (natural order in and out); w = W_A^m, m < A (used by A = 9).
template <int A, bool INV>
__device__ __forceinline__ void dft_odd(float2 (&x)[A], const float2 (&w)[A]) {
    if constexpr (A == 3) {
        dft3<INV>(x[0], x[1], x[2]);
    } else if constexpr (A == 5) {
        dft5<INV>(x[0], x[1], x[2], x[3], x[4]);
    } else if constexpr (A == 9) {   // 3 x 3 Cooley-Tukey: j = 3 j1 + j2, k = k1 + 3 k2
#pragma unroll
        for (int j2 = 0; j2 < 3; ++j2) dft3<INV>(x[j2], x[3 + j2], x[6 + j2]);   // x[3 k1 + j2] = y[j2][k1]
#pragma unroll
        for (int j2 = 1; j2 < 3; ++j2)
#pragma unroll
            for (int k1 = 1; k1 < 3; ++k1) x[3 * k1 + j2] = cmul<INV>(x[3 * k1 + j2], w[j2 * k1]);
        float2 y[9];
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            float2 a = x[3 * k1], b = x[3 * k1 + 1], c = x[3 * k1 + 2];
            dft3<INV>(a, b, c);
            y[k1] = a;
            y[k1 + 3] = b;
            y[k1 + 6] = c;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) x[k] = y[k];
    } else {   // A == 15: 3 x 5 Good-Thomas, j <-> (j mod 3, j mod 5), k = (5 k1 + 3 k2) mod 15
        static_assert(A == 15, "small odd DFTs: 3, 5, 9, 15");
        float2 z[15];   // z[5 k1 + j2]
#pragma unroll
        for (int j2 = 0; j2 < 5; ++j2) {
            // j = (10 j1 + 6 j2) mod 15 has j mod 3 = j1 and j mod 5 = j2
            float2 a = x[(6 * j2) % 15], b = x[(10 + 6 * j2) % 15], c = x[(20 + 6 * j2) % 15];
            dft3<INV>(a, b, c);
            z[j2] = a;
            z[5 + j2] = b;
            z[10 + j2] = c;
        }
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            float2* r = z + 5 * k1;
            dft5<INV>(r[0], r[1], r[2], r[3], r[4]);
#pragma unroll
            for (int k2 = 0; k2 < 5; ++k2) x[(5 * k1 + 3 * k2) % 15] = r[k2];
        }
    }
}

// x with (a * x) mod m == 1 (gcd(a, m) = 1), at compile time.
constexpr int mod_inverse(int a, int m) {
    for (int x = 1; x < m; ++x)
        if ((a * x) % m == 1) return x;
    return 1;
}

template <int A, int B>
struct Pfa {
    static constexpr int N = A * B, E = 16;
    static constexpr int TR = B / E;                      // threads per B-point sub-row
    static constexpr int T = A * TR;                      // threads per n-point row
    // Sub-row stride.  The load scatter sends lane i to bank pair (i + (i mod A)*SB) mod 16, a
    // permutation of the half-warp when SB is a multiple of 16; that is safe for the B-point
    // passes once a half-warp lies inside one sub-row (TR >= 16).  Narrower sub-rows keep the
    // exchange layout's own stride rule.
    static constexpr int SB = TR >= 16 ? (smem_stride<B, E, false>() + 15) / 16 * 16 : smem_stride<B, E, false>();
    static constexpr int ROWBUF = A * SB | 1;
    static constexpr int CTA = T < 256 ? (256 / T) * T : T;
    static constexpr int ROWS = CTA / T;
    static constexpr int COLS = (B + T - 1) / T;          // columns of the A-point phase per thread
    static constexpr int INV_B_MOD_A = mod_inverse(B % A, A);   // k1 = (k mod A) * B^-1 mod A
    static constexpr int INV_A_MOD_B = mod_inverse(A % B, B);   // k2 =  k * A^-1 mod B
    // n <= 12288: the A = 15, n = 15360 variant would need 960 threads and spills its columns
    static_assert(A % 2 == 1 && B % E == 0 && N <= (int)backend::kPfaMaxN, "shape outside the instantiated family");
};

template <int A, int B, bool INV>
__global__ void __launch_bounds__(Pfa<A, B>::CTA, min_blocks_64regs(Pfa<A, B>::CTA))
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

    // 1. coalesced loads, scattered to [j mod A][j mod B].  T is a multiple of A, so
    //    j mod A = tid mod A for every j = tid + i*T this thread loads.
    static_assert(T % A == 0, "the n-row team size is a multiple of A");
    {
        float2* rowA = buf + (tid % A) * P::SB;
#pragma unroll 4
        for (int i = 0; i < E; ++i) {
            const int j = tid + i * T;
            rowA[spad(j & (B - 1))] = ok ? ld_stream(src + j) : make_float2(0.f, 0.f);
        }
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
    // 3. A-point DFT down each column k2; X[(B k1 + A k2) mod n] = Y[k1][k2] kept at
    //    buf[k1*SB + k2] (unpadded: lanes hold consecutive k2, so the writes are contiguous)
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
            dft_odd<A, INV>(col[c], w);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) buf[k1 * P::SB + k2] = col[c][k1];
        }
    }
    __syncthreads();
    // 4. coalesced stores of X[k] = Y[k1][k2]; across lanes k2 steps by the odd A^-1 mod B,
    //    a permutation of the banks
    if (ok) {
        // k mod A = tid mod A for all k = tid + i*T, so k1 is fixed; k2 steps by T*A^-1 mod B
        const float2* rowK = buf + (((tid % A) * P::INV_B_MOD_A) % A) * P::SB;
        constexpr int STEP = (int)(((long long)T * P::INV_A_MOD_B) & (B - 1));
        int k2 = (tid * P::INV_A_MOD_B) & (B - 1);
#pragma unroll 4
        for (int i = 0; i < E; ++i) {
            st_stream(dst + tid + i * T, cscale(rowK[k2], scale));
            k2 = (k2 + STEP) & (B - 1);
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
