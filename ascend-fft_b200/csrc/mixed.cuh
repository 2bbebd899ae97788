// Mixed-radix Stockham kernels (device code shared by k_mixed.cu and the translation units
// that instantiate them: k_mixed_c0/c1/c2.cu for the runtime pass lists of each radix class,
// k_mixed_fixed.cu for the compile-time plans), and the host-side table type of one row
// policy's kernels.
// The algorithm: mixed-radix C2C for 13-smooth lengths (n = 2^a 3^b 5^c 7^d 11^e 13^f up to kMixedMaxN), one
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
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <initializer_list>
#include <tuple>

#include "backend.h"
#include "fft_kernels.cuh"
#include "fft_odd.cuh"
#include "istft_ola.cuh"

namespace bfly {
namespace dev {

struct MixedArgs {
    int n, passes;
    int radix[backend::kMixedMaxPasses];
    int ns[backend::kMixedMaxPasses];
    int twoff[backend::kMixedMaxPasses];
    unsigned magic[backend::kMixedMaxPasses];   // ceil(2^32 / ns), pass p >= 1
    // the buffer pass 0 writes: element i at i + i / pad0, pad0 = R_0 when R_0 is even (its
    // stride-R_0 stores then hit distinct banks), else 0 (element i at i); the other buffers
    // hold element i at spad(i)
    int pad0;
    unsigned magic0;   // ceil(2^32 / pad0), 0 when pad0 = 0
};

// KIND bit 0: source is the row in HBM (pass 0, which writes the pass-0 buffer); bit 1:
// destination is the row in HBM (scaled); bit 2: source is the pass-0 buffer (pass 1); bit 3:
// source is a row staged unpadded in shared memory (pass 0); bit 4: destination is shared
// memory, unpadded, in natural order (the last pass, for an epilogue).  Pass 0 (Ns = 1) has no
// twiddles.  The pass-0 buffer holds element i at i + i / pad0 (pad0 = R_0 or 0), computed once
// per butterfly: pass 0 stores j R_0 + r at j (R_0 + 1) + r, and pass 1 reads j + r nb (nb =
// n / R_1, a multiple of R_0) at j + j / R_0 + r (nb + nb / R_0).
template <int R, bool INV, int KIND>
__device__ __forceinline__ void mixed_pass(const float2* __restrict__ src, float2* __restrict__ dst, int n, int Ns,
                                           unsigned magic, const float2* __restrict__ twp, int t, int T,
                                           float scale, int pad0, unsigned magic0) {
    constexpr bool PASS0 = (KIND & 9) != 0;
    const int nb = n / R;
    const int nbs = (KIND & 4) ? nb + (int)__umulhi((unsigned)nb, magic0) : nb;
    const int stride0 = pad0 ? R + 1 : R;
    for (int j = t; j < nb; j += T) {
        const int k = PASS0 ? 0 : j - Ns * (int)__umulhi((unsigned)j, magic);
        const int js = (KIND & 4) ? j + (int)__umulhi((unsigned)j, magic0) : j;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
            v[r] = (KIND & 1)   ? ld_stream(src + j + r * nb)
                   : (KIND & 8) ? src[j + r * nb]
                   : (KIND & 4) ? src[js + r * nbs]
                                : src[spad(j + r * nb)];
        if (!PASS0) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul<INV>(v[r], __ldg(twp + (r - 1) * Ns + k));
        }
        DFT<R, INV>::run(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (KIND & 2) st_stream(dst + base + r * Ns, cscale(v[r], scale));
            else if (KIND & 16) dst[base + r * Ns] = v[r];
            else if (PASS0) dst[j * stride0 + r] = v[r];
            else dst[spad(base + r * Ns)] = v[r];
        }
    }
}

// Radix classes: CLS 0 compiles the radices up to 10, CLS 1 adds 12, 14, 15 and 16, CLS 2 the
// primes 11 and 13 (larger butterflies need more registers, and a kernel is allocated for its
// largest, so each plan runs the smallest class holding its radices).
template <bool INV, int KIND, int CLS>
__device__ __forceinline__ void mixed_pass_r(int R, const float2* src, float2* dst, int n, int Ns, unsigned magic,
                                             const float2* twp, int t, int T, float scale, int pad0,
                                             unsigned magic0) {
#define BFLY_MP(RR) \
    if (R == RR) return mixed_pass<RR, INV, KIND>(src, dst, n, Ns, magic, twp, t, T, scale, pad0, magic0)
    if constexpr (CLS >= 2) {
        BFLY_MP(13);
        BFLY_MP(11);
    }
    if constexpr (CLS >= 1) {
        BFLY_MP(16);
        BFLY_MP(15);
        BFLY_MP(14);
        BFLY_MP(12);
    }
    BFLY_MP(10);
    BFLY_MP(9);
    BFLY_MP(8);
    BFLY_MP(7);
    BFLY_MP(6);
    BFLY_MP(5);
    BFLY_MP(4);
    BFLY_MP(3);
#undef BFLY_MP
    mixed_pass<2, INV, KIND>(src, dst, n, Ns, magic, twp, t, T, scale, pad0, magic0);
}

// The passes of one row.  Pass 0 reads the row from HBM (SRC_HBM) or unpadded from buf1 (a
// stage written before the call); the last pass writes the row to HBM times `scale` (DST_HBM)
// or unpadded, natural order, into the buffer returned (buf0 or buf1).  All threads of the CTA
// call it (rows whose `ok` is false skip the work, not the barriers).
template <bool INV, int CLS, bool SRC_HBM, bool DST_HBM>
__device__ __forceinline__ float2* mixed_row(const MixedArgs& a, const float2* src, float2* dst, float2* buf0,
                                             float2* buf1, const float2* __restrict__ tw, bool ok, int t, int T,
                                             float scale) {
    constexpr int K0 = SRC_HBM ? 1 : 8;       // pass-0 source
    constexpr int KL = DST_HBM ? 2 : 16;      // last-pass destination
    const int n = a.n;
    float2* fin = buf0;
    for (int p = 0; p < a.passes; ++p) {
        const int R = a.radix[p], Ns = a.ns[p];
        const unsigned mg = a.magic[p];
        const float2* twp = tw + a.twoff[p];
        const bool first = p == 0, last = p == a.passes - 1;
        const float2* sb = (p & 1) ? buf0 : buf1;   // written by pass p - 1 (pass 0: the stage)
        float2* db = (p & 1) ? buf1 : buf0;
        float2* dl = DST_HBM ? dst : db;
        const int p0 = a.pad0;
        const unsigned m0 = a.magic0;
        if (ok) {
            if (first && last) mixed_pass_r<INV, K0 | KL, CLS>(R, SRC_HBM ? src : sb, dl, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (first) mixed_pass_r<INV, K0, CLS>(R, SRC_HBM ? src : sb, db, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (p == 1 && last) mixed_pass_r<INV, 4 | KL, CLS>(R, sb, dl, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (p == 1) mixed_pass_r<INV, 4, CLS>(R, sb, db, n, Ns, mg, twp, t, T, scale, p0, m0);
            else if (last) mixed_pass_r<INV, KL, CLS>(R, sb, dl, n, Ns, mg, twp, t, T, scale, p0, m0);
            else mixed_pass_r<INV, 0, CLS>(R, sb, db, n, Ns, mg, twp, t, T, scale, p0, m0);
        }
        if (last) fin = db;
        if (!last) __syncthreads();
    }
    return fin;
}

// The same passes for a plan fixed at compile time (its radices R0, R1, ...): n, Ns, the
// butterfly counts, threads per row and the pass-0 pad are constants, so the element offsets
// of every load and store fold into the instructions and the radix needs no dispatch.  T =
// min(512, ceil(n / R_max)) threads per row and pad0 = R_0 (even R_0) or 0, as mixedShape
// sets them; twiddles at the plan's offsets.
template <int R, bool INV, int KIND, int N, int NS, int T, int PAD0>
__device__ __forceinline__ void fixed_pass(const float2* __restrict__ src, float2* __restrict__ dst,
                                           const float2* __restrict__ twp, int t, float scale) {
    constexpr bool PASS0 = (KIND & 9) != 0;
    constexpr int nb = N / R;
    constexpr int nbs = (KIND & 4) && PAD0 ? nb + nb / PAD0 : nb;
    constexpr int stride0 = PAD0 ? R + 1 : R;
#pragma unroll
    for (int j0 = 0; j0 < nb; j0 += T) {
        const int j = j0 + t;
        if (nb % T != 0 && j >= nb) break;
        const int k = PASS0 ? 0 : j % NS;
        const int js = (KIND & 4) && PAD0 ? j + j / PAD0 : j;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
            v[r] = (KIND & 1)   ? ld_stream(src + j + r * nb)
                   : (KIND & 8) ? src[j + r * nb]
                   : (KIND & 4) ? src[js + r * nbs]
                                : src[spad(j + r * nb)];
        if (!PASS0) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul<INV>(v[r], __ldg(twp + (r - 1) * NS + k));
        }
        DFT<R, INV>::run(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (KIND & 2) st_stream(dst + base + r * NS, cscale(v[r], scale));
            else if (KIND & 16) dst[base + r * NS] = v[r];
            else if (PASS0) dst[j * stride0 + r] = v[r];
            else dst[spad(base + r * NS)] = v[r];
        }
    }
}

template <int... Rs>
struct FixedPlan {
    static constexpr int N = (Rs * ...);
    static constexpr int RMAX = std::max({Rs...});
    static constexpr int T = (N + RMAX - 1) / RMAX < 512 ? (N + RMAX - 1) / RMAX : 512;
    static constexpr int R0 = std::get<0>(std::make_tuple(Rs...));
    static constexpr int PAD0 = (R0 % 2 == 0 && sizeof...(Rs) > 1) ? R0 : 0;
};

template <bool INV, class FP, bool SRC_HBM, bool DST_HBM, int P, int NS, int R, int... Rest>
__device__ __forceinline__ float2* fixed_row(const float2* src, float2* dst, float2* buf0, float2* buf1,
                                             const float2* __restrict__ tw, const int* twoff, bool ok, int t,
                                             float scale) {
    constexpr bool LAST = sizeof...(Rest) == 0;
    constexpr int KIND = (P == 0 ? (SRC_HBM ? 1 : 8) : (P == 1 ? 4 : 0)) | (LAST ? (DST_HBM ? 2 : 16) : 0);
    const float2* sb = (P & 1) ? buf0 : buf1;
    float2* db = (P & 1) ? buf1 : buf0;
    if (ok)
        fixed_pass<R, INV, KIND, FP::N, NS, FP::T, FP::PAD0>(P == 0 && SRC_HBM ? src : sb, LAST && DST_HBM ? dst : db,
                                                            tw + twoff[P], t, scale);
    if constexpr (LAST) {
        return db;
    } else {
        __syncthreads();
        return fixed_row<INV, FP, SRC_HBM, DST_HBM, P + 1, NS * R, Rest...>(src, dst, buf0, buf1, tw, twoff, ok, t, scale);
    }
}

// Row policies of the kernels below: the runtime pass list (radix class CLS) or a plan fixed at
// compile time (Rs; launched with its T and pad0 only).
template <int CLS>
struct GenericRows {
    template <bool INV, bool SRC_HBM, bool DST_HBM>
    static __device__ __forceinline__ float2* run(const MixedArgs& a, const float2* src, float2* dst, float2* buf0,
                                                  float2* buf1, const float2* __restrict__ tw, bool ok, int t, int T,
                                                  float scale) {
        return mixed_row<INV, CLS, SRC_HBM, DST_HBM>(a, src, dst, buf0, buf1, tw, ok, t, T, scale);
    }
};
template <int... Rs>
struct FixedRows {
    template <bool INV, bool SRC_HBM, bool DST_HBM>
    static __device__ __forceinline__ float2* run(const MixedArgs& a, const float2* src, float2* dst, float2* buf0,
                                                  float2* buf1, const float2* __restrict__ tw, bool ok, int t, int,
                                                  float scale) {
        return fixed_row<INV, FixedPlan<Rs...>, SRC_HBM, DST_HBM, 0, 1, Rs...>(src, dst, buf0, buf1, tw, a.twoff, ok, t,
                                                                             scale);
    }
};

template <bool INV, class ROWS>
__global__ void __launch_bounds__(512, 2) k_mixed(const float2* __restrict__ in, float2* __restrict__ out,
                                                  const float2* __restrict__ tw, MixedArgs a, uint64_t batch, int T,
                                                  int rows, int len, float scale) {
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * rows + rl;
    const bool ok = rl < rows && row < batch;
    float2* buf0 = smem + (size_t)(rl < rows ? rl : 0) * 2 * len;
    ROWS::template run<INV, true, true>(a, in + row * a.n, out + row * a.n, buf0, buf0 + len, tw, ok, t, T, scale);
}

// Real transforms of even length N = 2M on the mixed-radix passes of the M-point complex row
// (M 13-smooth).  twr[k] = W_N^k, k <= M.
// R2C (numpy.fft.rfft): z[m] = x[2m] + i x[2m+1] read as complex, Z = FFT_M(z) left unpadded in
// shared memory, then per bin k <= M: a = Z[k mod M], b = conj(Z[(M-k) mod M]),
// X[k] = (a+b)/2 + W_N^k (a-b)/(2i), times s_edge at bins 0 and M and s_int elsewhere.
template <class ROWS>
__global__ void __launch_bounds__(512, 2) k_r2c_mixed(const float2* __restrict__ in, float2* __restrict__ out,
                                                      const float2* __restrict__ tw, const float2* __restrict__ twr,
                                                      MixedArgs a, uint64_t batch, int T, int rows, int len,
                                                      float s_edge, float s_int) {
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * rows + rl;
    const bool ok = rl < rows && row < batch;
    const int M = a.n;
    float2* buf0 = smem + (size_t)(rl < rows ? rl : 0) * 2 * len;
    const float2* Z = ROWS::template run<false, true, false>(a, in + row * M, nullptr, buf0, buf0 + len, tw, ok, t, T,
                                                           1.f);
    __syncthreads();
    if (!ok) return;
    float2* dst = out + row * (uint64_t)(M + 1);
    for (int k = t; k <= M; k += T) {
        const float2 za = Z[k < M ? k : 0];
        const float2 zb = Z[k > 0 ? M - k : 0];
        const float2 e = make_float2(0.5f * (za.x + zb.x), 0.5f * (za.y - zb.y));
        const float2 o = make_float2(0.5f * (za.y + zb.y), 0.5f * (zb.x - za.x));
        const float2 X = cadd(e, cmul<false>(o, __ldg(twr + k)));
        st_stream(dst + k, cscale(X, (k == 0 || k == M) ? s_edge : s_int));
    }
}

// C2R (numpy.fft.irfft when out_scale = 1/N, as k_c2r): the un-split spectrum
// Z[k] = (Xk + conj Xm) + i (Xk - conj Xm) W_N^-k (Xm = X[M-k], X[M] for k = 0; imaginary parts of
// bins 0 and M ignored; s_edge / s_int per bin; out_scale) is staged unpadded in shared memory,
// then z = IFFT_M(Z) goes to HBM as x[2m] = Re z[m], x[2m+1] = Im z[m].
template <class ROWS>
__global__ void __launch_bounds__(512, 2) k_c2r_mixed(const float2* __restrict__ in, float2* __restrict__ out,
                                                      const float2* __restrict__ tw, const float2* __restrict__ twr,
                                                      MixedArgs a, uint64_t batch, int T, int rows, int len,
                                                      float s_edge, float s_int, float out_scale) {
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * rows + rl;
    const bool ok = rl < rows && row < batch;
    const int M = a.n;
    float2* buf0 = smem + (size_t)(rl < rows ? rl : 0) * 2 * len;
    float2* buf1 = buf0 + len;
    const float2* src = in + row * (uint64_t)(M + 1);
    if (ok)
        for (int k = t; k < M; k += T)
            buf1[k] = c2r_split(ld_stream(src + k), ld_stream(src + (k == 0 ? M : M - k)), k, __ldg(twr + k), s_edge,
                                s_int, out_scale);
    __syncthreads();
    ROWS::template run<true, false, true>(a, nullptr, out + row * M, buf0, buf1, tw, ok, t, T, 1.f);
}

// STFT: frame f of signal s, y[j] = w[j] x_s[f hop + j - (center ? N/2 : 0)] (reflect padding,
// as k_stft), packed as z[m] = y[2m] + i y[2m+1] and staged unpadded; then the R2C of k_r2c_mixed.
template <class ROWS>
__global__ void __launch_bounds__(512, 2) k_stft_mixed(const float* __restrict__ sig, float2* __restrict__ out,
                                                       const float2* __restrict__ tw, const float2* __restrict__ twr,
                                                       const float* __restrict__ window, MixedArgs a, uint64_t frames,
                                                       uint32_t framesPerSignal, int64_t sigLen, uint64_t sigStride,
                                                       uint32_t hop, int center, int T, int rows, int len) {
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * rows + rl;
    const bool ok = rl < rows && row < frames;
    const int M = a.n;
    float2* buf0 = smem + (size_t)(rl < rows ? rl : 0) * 2 * len;
    float2* buf1 = buf0 + len;
    if (ok) {
        const uint64_t s = row / framesPerSignal, f = row % framesPerSignal;
        const float* x = sig + s * sigStride;
        const int64_t start = (int64_t)f * hop - (center ? M : 0);
        auto sample = [&](int64_t i) {
            i = i < 0 ? -i : i;
            i = i >= sigLen ? 2 * (sigLen - 1) - i : i;
            return __ldg(x + i);
        };
        // interior frames starting on an 8-byte boundary read one float2 per complex value; the
        // others sample with reflection
        const bool direct = start >= 0 && start + 2 * M <= sigLen && (reinterpret_cast<uintptr_t>(x + start) & 7u) == 0;
        const float2* xv = reinterpret_cast<const float2*>(x + (direct ? start : 0));
        const float2* wv = reinterpret_cast<const float2*>(window);
        for (int m = t; m < M; m += T) {
            float2 z = direct ? __ldg(xv + m) : make_float2(sample(start + 2 * m), sample(start + 2 * m + 1));
            if (window) {
                const float2 w = __ldg(wv + m);
                z = make_float2(z.x * w.x, z.y * w.y);
            }
            buf1[m] = z;
        }
    }
    __syncthreads();
    const float2* Z = ROWS::template run<false, false, false>(a, nullptr, nullptr, buf0, buf1, tw, ok, t, T, 1.f);
    __syncthreads();
    if (!ok) return;
    float2* dst = out + row * (uint64_t)(M + 1);
    for (int k = t; k <= M; k += T) {
        const float2 za = Z[k < M ? k : 0];
        const float2 zb = Z[k > 0 ? M - k : 0];
        const float2 e = make_float2(0.5f * (za.x + zb.x), 0.5f * (za.y - zb.y));
        const float2 o = make_float2(0.5f * (za.y + zb.y), 0.5f * (zb.x - za.x));
        st_stream(dst + k, cadd(e, cmul<false>(o, __ldg(twr + k))));
    }
}

// Inverse STFT of even non-power-of-two N = 2M (M 13-smooth) in one kernel: per wave each row
// stages its frame's un-split spectrum (c2r_split, out_scale) in buf1 and runs the M-point
// inverse passes into its natural-order row buffer; the segment split, carry, envelope and
// overlap-add (window applied there) are IstftSegment (istft_ola.cuh), as in k_istft.
template <class ROWS, int VEC>
__global__ void __launch_bounds__(512, 2) k_istft_mixed(const float2* __restrict__ spec, float* __restrict__ out,
                                                        const float2* __restrict__ tw, const float2* __restrict__ twr,
                                                        const float* __restrict__ window, MixedArgs a, uint32_t frames,
                                                        uint32_t hop, uint32_t Q, uint32_t segs, int64_t start,
                                                        uint64_t outLen, float out_scale, int T, int rows, int len) {
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const int M = a.n;
    IstftSegment seg;
    seg.init(2 * M, hop, frames, Q, segs, start, outLen, window, out,
             reinterpret_cast<float*>(smem + (size_t)rows * 2 * len));
    const float2* src0 = spec + (uint64_t)(blockIdx.x / segs) * frames * (M + 1);
    float2* buf0 = smem + (size_t)rl * 2 * len;
    float2* buf1 = buf0 + len;
    const int finOff = ((a.passes - 1) & 1) ? len : 0;   // buffer the last pass writes
    auto frameOf = [&](int r) { return reinterpret_cast<const float*>(smem + (size_t)r * 2 * len + finOff); };

    for (uint32_t f0 = seg.fA; f0 < seg.fB; f0 += rows) {
        const int R = (int)min((uint32_t)rows, seg.fB - f0);
        __syncthreads();   // the previous wave is done with the row buffers and the carry
        // rows past R (a CTA's partial first or last wave) transform frame f0 again, unread
        const float2* src = src0 + (uint64_t)(f0 + (rl < R ? rl : 0)) * (M + 1);
        for (int k = t; k < M; k += T)
            buf1[k] = c2r_split(ld_stream(src + k), ld_stream(src + (k == 0 ? M : M - k)), k, __ldg(twr + k), 1.f, 1.f,
                                out_scale);
        __syncthreads();
        ROWS::template run<true, false, false>(a, nullptr, nullptr, buf0, buf1, tw, true, t, T, 1.f);
        __syncthreads();
        seg.wave<VEC, 0>(
            f0, R, [&](int r, int j) { return (window ? __ldg(window + j) : 1.f) * frameOf(r)[j]; },
            [&](int r, int j) {
                const float4 x = *reinterpret_cast<const float4*>(frameOf(r) + j);
                const float4 w = window ? __ldg(reinterpret_cast<const float4*>(window + j)) : make_float4(1.f, 1.f, 1.f, 1.f);
                return make_float4(w.x * x.x, w.y * x.y, w.z * x.z, w.w * x.w);
            });
    }
    seg.zeroTail(segs);
}

}  // namespace dev

namespace backend {
// The kernels of one row policy.
using C2CFn = decltype(&dev::k_mixed<false, dev::GenericRows<0>>);
using R2CFn = decltype(&dev::k_r2c_mixed<dev::GenericRows<0>>);
using C2RFn = decltype(&dev::k_c2r_mixed<dev::GenericRows<0>>);
using StftFn = decltype(&dev::k_stft_mixed<dev::GenericRows<0>>);
using IstftFn = decltype(&dev::k_istft_mixed<dev::GenericRows<0>, 1>);
struct MixedKernels {
    C2CFn fwd, inv;
    R2CFn r2c;
    C2RFn c2r;
    StftFn stft;
    IstftFn istft1, istft4;
};
template <class ROWS>
MixedKernels kernelsOf() {
    return {dev::k_mixed<false, ROWS>, dev::k_mixed<true, ROWS>, dev::k_r2c_mixed<ROWS>, dev::k_c2r_mixed<ROWS>,
            dev::k_stft_mixed<ROWS>, dev::k_istft_mixed<ROWS, 1>, dev::k_istft_mixed<ROWS, 4>};
}

// Plans with compile-time kernels (common lengths: multiples of 10 and the half lengths of the
// real transforms of n = 400, 480, 1000, 2000, 6000 ...); every other plan runs the runtime
// pass list of its radix class.
struct FixedEntry {
    int passes;
    int radix[5];
    int T, pad0;   // the shape the kernels are compiled for
    MixedKernels k;
};
#define BFLY_FIXED(...)                                                                              \
    {(int)std::initializer_list<int>{__VA_ARGS__}.size(), {__VA_ARGS__}, dev::FixedPlan<__VA_ARGS__>::T, \
     dev::FixedPlan<__VA_ARGS__>::PAD0, kernelsOf<dev::FixedRows<__VA_ARGS__>>()}

// The kernels of the runtime pass lists of radix class 0, 1, 2 (k_mixed_c0/c1/c2.cu) and the
// table of compile-time plans (k_mixed_fixed.cu).
MixedKernels mixedGeneric0();
MixedKernels mixedGeneric1();
MixedKernels mixedGeneric2();
const FixedEntry* mixedFixed(int* count);
}  // namespace backend
}  // namespace bfly
