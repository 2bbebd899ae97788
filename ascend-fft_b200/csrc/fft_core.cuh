// Device core of the batched power-of-two FFT: in-register DFTs of size 2/4/8/16, the
// Stockham autosort pass schedule, and the "team" FFT in which T = N/E threads each hold
// E complex values and exchange them through padded shared memory between passes.
//
// Transform computed (forward): X[k] = sum_j x[j] * exp(-2*pi*i*j*k/N), unnormalised, the
// convention of the reference's Plan::run (src/framework/butterfly.cpp:723-749, kernel
// src/ascendc/fft_radix2.cpp:51).  INV flips the exponent sign (unnormalised inverse).
//
// Pass p of the schedule has radix R_p and Ns_p = R_0*...*R_{p-1}.  Butterfly j (0 <= j < N/R_p)
// with k = j mod Ns_p reads x[j + r*N/R_p] (r < R_p), multiplies element r by
// exp(-2*pi*i*r*k/(Ns_p*R_p)), applies DFT_{R_p} and writes y[(j-k)*R_p + k + r*Ns_p].
// Reads are unit-stride across threads in every pass, and the last pass writes
// y[j + r*N/R_last], so first-pass loads and last-pass stores are coalesced global accesses.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bfly {
namespace dev {

// ------------------------------------------------------------------ complex helpers
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// a * w (CONJ=false) or a * conj(w) (CONJ=true)
template <bool CONJ>
__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
    if (CONJ) return make_float2(fmaf(a.x, w.x, a.y * w.y), fmaf(a.y, w.x, -(a.x * w.y)));
    return make_float2(fmaf(a.x, w.x, -(a.y * w.y)), fmaf(a.x, w.y, a.y * w.x));
}

// Multiply by exp(-2*pi*i*q/16) for a compile-time q (forward direction). Exact special cases
// for multiples of pi/4; the remaining angles use correctly rounded constants.
template <int Q>
__device__ __forceinline__ float2 rot16(float2 a) {
    constexpr int q = ((Q % 16) + 16) % 16;
    constexpr float H = 0.70710678118654752440f;   // sqrt(1/2)
    constexpr float C1 = 0.92387953251128675613f;  // cos(pi/8)
    constexpr float S1 = 0.38268343236508977173f;  // sin(pi/8)
    if constexpr (q == 0) return a;
    else if constexpr (q == 4) return make_float2(a.y, -a.x);
    else if constexpr (q == 8) return make_float2(-a.x, -a.y);
    else if constexpr (q == 12) return make_float2(-a.y, a.x);
    else if constexpr (q == 2) return make_float2(H * (a.x + a.y), H * (a.y - a.x));
    else if constexpr (q == 6) return make_float2(H * (a.y - a.x), -H * (a.x + a.y));
    else if constexpr (q == 10) return make_float2(-H * (a.x + a.y), H * (a.x - a.y));
    else if constexpr (q == 14) return make_float2(H * (a.x - a.y), H * (a.x + a.y));
    else {
        // cos/sin of 2*pi*q/16 for odd q
        constexpr float c = (q == 1 || q == 15) ? C1 : (q == 3 || q == 13) ? S1
                          : (q == 5 || q == 11) ? -S1 : -C1;
        constexpr float s = (q == 1 || q == 7) ? S1 : (q == 3 || q == 5) ? C1
                          : (q == 9 || q == 15) ? -S1 : -C1;
        // a * (c - i s)
        return make_float2(fmaf(a.x, c, a.y * s), fmaf(a.y, c, -(a.x * s)));
    }
}

// a * exp(sign*2*pi*i*e/R), sign = -1 forward, +1 inverse; R divides 16.
template <int E, int R, bool INV>
__device__ __forceinline__ float2 rot(float2 a) {
    constexpr int q = (16 / R) * E;
    if constexpr (INV) return rot16<16 - (q % 16)>(a);
    else return rot16<q>(a);
}

// ------------------------------------------------------------------ in-register DFTs
// Natural order in and out: v[k] <- sum_m v[m] * exp(sign*2*pi*i*m*k/R).
template <int R, bool INV> struct DFT;

template <bool INV> struct DFT<1, INV> {
    static __device__ __forceinline__ void run(float2*) {}
};

template <bool INV> struct DFT<2, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        const float2 a = v[0];
        v[0] = cadd(a, v[1]);
        v[1] = csub(a, v[1]);
    }
};

template <bool INV> struct DFT<4, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        const float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        const float2 t2 = cadd(v[1], v[3]);
        float2 t3 = csub(v[1], v[3]);
        t3 = INV ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);  // * (+-i)
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    }
};

template <int A, int B, int R, bool INV, int K1 = 0, int N2 = 0>
__device__ __forceinline__ void twiddle_split_impl(float2* v) {
    if constexpr (K1 < A) {
        if constexpr (N2 < B) {
            v[B * K1 + N2] = rot<K1 * N2, R, INV>(v[B * K1 + N2]);
            twiddle_split_impl<A, B, R, INV, K1, N2 + 1>(v);
        } else {
            twiddle_split_impl<A, B, R, INV, K1 + 1, 0>(v);
        }
    }
}
template <int A, int B, int R, bool INV>
__device__ __forceinline__ void twiddle_split(float2* v) { twiddle_split_impl<A, B, R, INV>(v); }

// R = A*B Cooley-Tukey in registers. Input n = B*n1 + n2, output k = k1 + A*k2.
template <int A, int B, bool INV>
__device__ __forceinline__ void dft_split(float2* v) {
    constexpr int R = A * B;
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
        float2 col[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) col[n1] = v[B * n1 + n2];
        DFT<A, INV>::run(col);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) v[B * k1 + n2] = col[k1];
    }
    // twiddles w_R^(n2*k1): unrolled with compile-time exponents
    twiddle_split<A, B, R, INV>(v);
    float2 out[R];
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
        float2 row[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) row[n2] = v[B * k1 + n2];
        DFT<B, INV>::run(row);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) out[k1 + A * k2] = row[k2];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = out[i];
}

template <bool INV> struct DFT<8, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_split<2, 4, INV>(v); }
};
template <bool INV> struct DFT<16, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_split<4, 4, INV>(v); }
};

// ------------------------------------------------------------------ pass schedule
// Greedy radix schedule: radix E while it divides the remaining length, remainder last.
// Shared with the host twiddle-table builder through the same constexpr functions.
__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

template <int N, int E>
struct Sched {
    static_assert((N & (N - 1)) == 0 && N >= 2, "N must be a power of two");
    static_assert(E == 2 || E == 4 || E == 8 || E == 16, "E must be 2,4,8,16");
    static_assert(N >= E, "N must be >= E");
    static constexpr int T = N / E;                      // threads per transform
    static constexpr int LOGN = ilog2c(N), LOGE = ilog2c(E);
    static constexpr int P = (LOGN + LOGE - 1) / LOGE;   // number of passes
    __host__ __device__ static constexpr int radix(int p) {
        return (p < P - 1) ? E : (1 << (LOGN - (P - 1) * LOGE));
    }
    __host__ __device__ static constexpr int ns(int p) {  // product of radices before p
        int v = 1;
        for (int q = 0; q < p; ++q) v *= radix(q);
        return v;
    }
    // float2 offset of pass p's twiddles in the table: (R_p - 1) * Ns_p entries per pass p >= 1
    __host__ __device__ static constexpr int twoff(int p) {
        int off = 0;
        for (int q = 1; q < p; ++q) off += (radix(q) - 1) * ns(q);
        return off;
    }
    static constexpr int TWSIZE = twoff(P);
};

// Shared-memory layout: one pad element per 16 (8-byte words => 16 banks of a half-warp).
__host__ __device__ constexpr int spad(int i) { return i + (i >> 4); }

// Row stride (in float2) of one transform's exchange buffer.
//  ROW_FAST=false: lanes of a half-warp are consecutive threads t of the same transform
//    (or, when T < 16, of 16/T consecutive transforms): stride = T mod 16 keeps the
//    transforms in disjoint bank groups.
//  ROW_FAST=true : lanes are consecutive transforms with the same t: an odd stride spreads
//    them over all 16 banks whatever the within-transform index.
template <int N, int E, bool ROW_FAST>
__host__ __device__ constexpr int smem_stride() {
    constexpr int base = spad(N - 1) + 1;
    constexpr int T = N / E;
    if constexpr (ROW_FAST) return base | 1;
    else if constexpr (T < 16) return base + ((T - (base % 16)) % 16 + 16) % 16;
    else return base;
}

// ------------------------------------------------------------------ synchronisation
// How the threads of one transform synchronise between passes:
//   kSyncWarp   the transform lives inside one warp (T <= 32)
//   kSyncNamed  the transform spans whole warps of a larger CTA: named barrier 1 + row, T threads
//   kSyncBlock  the transform is the whole CTA
enum SyncKind { kSyncWarp = 0, kSyncNamed = 1, kSyncBlock = 2 };

template <int SYNC>
__device__ __forceinline__ void team_sync(int row, int nthreads) {
    if constexpr (SYNC == kSyncWarp) {
        __syncwarp();
    } else if constexpr (SYNC == kSyncNamed) {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + row), "r"(nthreads) : "memory");
    } else {
        __syncthreads();
    }
}

// Sync policy for a transform of T threads in a CTA of `ctaThreads`.
__host__ __device__ constexpr int sync_kind(int T, int ctaThreads) {
    return T <= 32 ? kSyncWarp : (T < ctaThreads ? kSyncNamed : kSyncBlock);
}

// ------------------------------------------------------------------ team FFT
// One transform of length N held by T = N/E threads, E complex values per thread.
// Thread t, slot s (< E/R), element r of pass p covers butterfly j = t + s*T.
// On return, v[s*R_last + r] holds output element t + s*T + r*(N/R_last) (natural order).
// `sm` is this transform's exchange buffer (smem_stride<> float2), `tw` the Stockham
// twiddle table of Sched<N,E> (TWSIZE entries, pass p at twoff(p)), `load(i)` yields input
// element i.  SYNC selects the barrier (see team_sync); `row` is the transform's index in its
// CTA (named-barrier id - 1).  ESTRIDE selects the exchange layout: 0 = element i at
// sm[spad(i)] (padded, threads of one transform across lanes); s > 0 = element i at sm[i*s]
// (transforms across lanes, e.g. the columns of a tile staged densely by TMA).
template <int N, int E, bool INV, int SYNC, int ESTRIDE = 0>
struct Team {
    using S = Sched<N, E>;
    static constexpr int T = S::T;
    static constexpr int P = S::P;

    static __device__ __forceinline__ int at(int i) {
        if constexpr (ESTRIDE == 0) return spad(i);
        else return i * ESTRIDE;
    }

    static __device__ __forceinline__ void sync(int row) { team_sync<SYNC>(row, T); }

    template <class Load>
    static __device__ __forceinline__ void load_first(float2 (&v)[E], int t, Load&& load) {
        constexpr int R = S::radix(0);
        constexpr int B = E / R;
#pragma unroll
        for (int s = 0; s < B; ++s)
#pragma unroll
            for (int r = 0; r < R; ++r) v[s * R + r] = load(t + s * T + r * (N / R));
    }

    template <int p>
    static __device__ __forceinline__ void passes(float2 (&v)[E], float2* sm,
                                                  const float2* __restrict__ tw, int t, int row) {
        constexpr int R = S::radix(p);
        constexpr int B = E / R;
        constexpr int Ns = S::ns(p);
        if constexpr (p > 0) {
            const float2* twp = tw + S::twoff(p);
#pragma unroll
            for (int s = 0; s < B; ++s) {
                const int k = (t + s * T) & (Ns - 1);
#pragma unroll
                for (int r = 1; r < R; ++r)
                    v[s * R + r] = cmul<INV>(v[s * R + r], __ldg(twp + (r - 1) * Ns + k));
            }
        }
#pragma unroll
        for (int s = 0; s < B; ++s) DFT<R, INV>::run(&v[s * R]);
        if constexpr (p < P - 1) {
#pragma unroll
            for (int s = 0; s < B; ++s) {
                const int j = t + s * T;
                const int k = j & (Ns - 1);
                const int base = (j - k) * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) sm[at(base + r * Ns)] = v[s * R + r];
            }
            sync(row);
            constexpr int R2 = S::radix(p + 1);
            constexpr int B2 = E / R2;
#pragma unroll
            for (int s = 0; s < B2; ++s)
#pragma unroll
                for (int r = 0; r < R2; ++r) v[s * R2 + r] = sm[at(t + s * T + r * (N / R2))];
            if constexpr (p + 1 < P - 1) sync(row);   // next pass writes the buffer again
            passes<p + 1>(v, sm, tw, t, row);
        }
    }

    // Element index held in v[s*R_last + r] after run().
    static __device__ __forceinline__ int out_index(int t, int s, int r) {
        constexpr int R = S::radix(P - 1);
        return t + s * T + r * (N / R);
    }

    template <class Load>
    static __device__ __forceinline__ void run(float2 (&v)[E], float2* sm,
                                               const float2* __restrict__ tw, int t, int row,
                                               Load&& load) {
        load_first(v, t, load);
        passes<0>(v, sm, tw, t, row);
    }

    // Apply f(index, value&) to every output element held by this thread (in place).
    template <class F>
    static __device__ __forceinline__ void for_each_slot(float2 (&v)[E], int t, F&& f) {
        constexpr int R = S::radix(P - 1);
        constexpr int B = E / R;
#pragma unroll
        for (int s = 0; s < B; ++s)
#pragma unroll
            for (int r = 0; r < R; ++r) f(t + s * T + r * (N / R), v[s * R + r]);
    }

    // Apply f(index, value) to every output element held by this thread.
    template <class F>
    static __device__ __forceinline__ void for_each_out(float2 (&v)[E], int t, F&& f) {
        constexpr int R = S::radix(P - 1);
        constexpr int B = E / R;
#pragma unroll
        for (int s = 0; s < B; ++s)
#pragma unroll
            for (int r = 0; r < R; ++r) f(t + s * T + r * (N / R), v[s * R + r]);
    }
};

// ------------------------------------------------------------------ programmatic dependent launch
// A kernel launched with programmatic stream serialisation may start while the previous kernel
// on its stream drains: pdl_wait(), before a kernel's first global access, blocks until the
// previous grid has finished and its writes are visible, so a chain of such launches overlaps
// only launch latency, never data; pdl_trigger(), just before a CTA's final stores, lets the
// next kernel launch once every CTA of this grid has reached that point (triggering at entry
// placed the next grid's CTAs beside this one's and unbalanced one-wave launches).  Without
// the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ------------------------------------------------------------------ global access helpers
// Streaming (evict-first) accesses: every input and output element is touched exactly once.
__device__ __forceinline__ float2 ld_stream(const float2* p) { return __ldcs(p); }
// Input load with the default cache operator (ld.global.ca, a coherent weak load, valid for
// inputs written by a kernel that a programmatic-launch wait ordered before this one).  On the
// single-length C2C kernel it measured 2 % faster than evict-first loads with N(0,1) inputs
// (n = 4096: 0.846 -> 0.861 of the copy peak at batch 4096, 0.896 -> 0.914 at 8192), level
// with read-only (.nc) loads, which are not used because an input may be written by a kernel
// still draining when this one launches.  The two four-step passes gained too (long C2C
// n = 32768: 0.433 -> 0.455; 65536: 0.443 -> 0.446) and so did the column pass (NY = 1024:
// 0.57 -> 0.59); R2C, C2R, the mixed-radix, prime-factor, STFT and Bluestein kernels measured level.  Kernels that
// keep several twiddle tables in L1 (the ragged launch over many lengths) lost with it and keep
// ld_stream.
__device__ __forceinline__ float2 ld_once_ca(const float2* p) { return __ldca(p); }
__device__ __forceinline__ void st_stream(float2* p, float2 v) { __stcs(p, v); }

}  // namespace dev
}  // namespace bfly
