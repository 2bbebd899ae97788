// Kernel templates of the batched FFT library (sm_100a).
//
//   k_c2c      batched C2C, one team per row, rows [batch][N] interleaved fp32.
//              Reference: Plan::run -> kfft_fwd (src/framework/butterfly.cpp:723-749,
//              src/ascendc/fft_radix2.cpp:51-481).
//   k_r2c      R2C as an N/2 complex FFT with the even/odd split fused into its epilogue;
//              writes the dense half spectrum [batch][N/2+1] complex (= [batch][N+2] floats).
//              Reference: Plan::runR2C -> kfft_fwd(n/2) + kfft_r2c_post
//              (butterfly.cpp:753-806, src/ascendc/fft_real.cpp:47-162).
//   k_c2r      C2R as an N/2 complex inverse with the Hermitian un-split fused into its
//              prologue; output includes 1/N like numpy.fft.irfft.
//              Reference: Plan::runC2R -> kfft_c2r_prep + kfft_fwd(xflip) + kfft_c2r_post
//              (butterfly.cpp:810-850, fft_real.cpp:167-267).
//   k_long_a / k_long_b
//              four-step long C2C, N = N1*N2: column FFTs of N1 with the W_N^(n2*k1) twiddle
//              fused into the store, then row FFTs of N2 with the transpose fused into the
//              store.  Reference: four-step chain of src/host/fft_check.cpp:289-308, 843-970,
//              kfft_lt_tr / kfft_lt_tw (src/ascendc/fft_long_lt_tr.inc:22-157,
//              src/ascendc/fft_long.cpp:82-140).
//   k_tw_*     twiddle tables computed in FP64 on the GPU and rounded to fp32.
#pragma once
#include "fft_core.cuh"

namespace bfly {
namespace dev {

// ------------------------------------------------------------------ C2C
// Minimum resident CTAs that keeps a kernel at <= 64 registers per thread: the budget at which
// the 512-thread single-transform kernels still fit two CTAs per SM.
__host__ __device__ constexpr int min_blocks_64regs(int threads) {
    return 65536 / (threads * 64) > 0 ? 65536 / (threads * 64) : 1;
}

template <int N, int E, int ROWS, bool INV>
__global__ void __launch_bounds__((N / E) * ROWS, min_blocks_64regs((N / E) * ROWS))
k_c2c(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
      uint64_t batch, float scale) {
    constexpr int T = N / E;
    constexpr int S = smem_stride<N, E, false>();
    using TM = Team<N, E, INV, sync_kind(T, T * ROWS)>;
    extern __shared__ float2 smem[];
    pdl_wait();
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * ROWS + rl;
    const bool ok = row < batch;
    const float2* src = in + row * N;
    float2* dst = out + row * N;
    float2 v[E];
    TM::run(v, smem + rl * S, tw, t, rl,
            [&](int i) { return ok ? ld_once_ca(src + i) : make_float2(0.f, 0.f); });
    pdl_trigger();
    if (ok) TM::for_each_out(v, t, [&](int i, float2 x) { st_stream(dst + i, cscale(x, scale)); });
}

// ------------------------------------------------------------------ R2C
// x real [N] viewed as z[m] = x[2m] + i x[2m+1] (M = N/2), Z = FFT_M(z), then for k = 0..M:
//   a = Z[k mod M], b = conj(Z[(M-k) mod M]), E = (a+b)/2, O = (a-b)/(2i),
//   X[k] = E + W_N^k O.          (same split as fft_real.cpp:9-14, :139-149)
// Optional per-bin weights (WEIGHTED): X[k] *= (k==0||k==M ? s_edge : s_int); used by the
// adjoint of C2R.
template <int N, int E, int ROWS, bool WEIGHTED>
__global__ void __launch_bounds__((N / 2 / E) * ROWS, min_blocks_64regs((N / 2 / E) * ROWS))
k_r2c(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
      const float2* __restrict__ twr, uint64_t batch, float s_edge, float s_int) {
    constexpr int M = N / 2;
    constexpr int T = M / E;
    constexpr int S = smem_stride<M, E, false>();
    using TM = Team<M, E, false, sync_kind(T, T * ROWS)>;
    extern __shared__ float2 smem[];
    pdl_wait();
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * ROWS + rl;
    const bool ok = row < batch;
    const float2* src = in + row * M;
    float2* dst = out + row * (M + 1);
    float2* sm = smem + rl * S;
    float2 v[E];
    TM::run(v, sm, tw, t, rl, [&](int i) { return ok ? ld_stream(src + i) : make_float2(0.f, 0.f); });
    // twiddles of this thread's output bins k = t + i*T (and bin M for t == 0), in flight
    // while Z goes through shared memory
    float2 w[E];
#pragma unroll
    for (int i = 0; i < E; ++i) w[i] = __ldg(twr + t + i * T);
    const float2 wm = __ldg(twr + M);
    TM::sync(rl);
    TM::for_each_out(v, t, [&](int i, float2 x) { sm[spad(i)] = x; });
    TM::sync(rl);
    pdl_trigger();
    if (!ok) return;
    auto bin = [&](int k, float2 wk) {
        const float2 a = sm[spad(k & (M - 1))];
        const float2 b = sm[spad((M - k) & (M - 1))];
        const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
        const float2 o = make_float2(0.5f * (a.y + b.y), 0.5f * (b.x - a.x));
        float2 X = cadd(e, cmul<false>(o, wk));
        if constexpr (WEIGHTED) X = cscale(X, (k == 0 || k == M) ? s_edge : s_int);
        st_stream(dst + k, X);
    };
#pragma unroll
    for (int i = 0; i < E; ++i) bin(t + i * T, w[i]);
    if (t == 0) bin(M, wm);
}

// ------------------------------------------------------------------ C2R
// X half spectrum [M+1] (M = N/2), staged once in shared memory.  Imaginary parts of X[0] and
// X[M] are ignored, as in the real part extraction of kfft_c2r_post (fft_real.cpp:262-263).
// For k = 0..M-1:
//   Xk = X[k], Xm = X[M-k] (scaled by s_edge at DC/Nyquist, s_int elsewhere),
//   Z[k] = (Xk + conj Xm) + i (Xk - conj Xm) W_N^-k,  z = IDFT_M(Z) * out_scale,
//   x[2m] = Re z[m], x[2m+1] = Im z[m].   out_scale = 1/N gives numpy.fft.irfft.
// C2R split of bin k: xk = X[k], xm = X[M-k] (xm = X[M] for k = 0), twk = W_N^k.
__device__ __forceinline__ float2 c2r_split(float2 xk, float2 xm, int k, float2 twk, float s_edge, float s_int,
                                            float out_scale) {
    if (k == 0) {
        xk = make_float2(xk.x * s_edge, 0.f);
        xm = make_float2(xm.x * s_edge, 0.f);
    } else {
        xk = cscale(xk, s_int);
        xm = cscale(xm, s_int);
    }
    const float2 ev = make_float2(xk.x + xm.x, xk.y - xm.y);
    const float2 od = cmul<true>(make_float2(xk.x - xm.x, xk.y + xm.y), twk);
    return make_float2((ev.x - od.y) * out_scale, (ev.y + od.x) * out_scale);
}

template <int N, int E, int ROWS>
__global__ void __launch_bounds__((N / 2 / E) * ROWS, min_blocks_64regs((N / 2 / E) * ROWS))
k_c2r(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
      const float2* __restrict__ twr, uint64_t batch, float s_edge, float s_int, float out_scale) {
    constexpr int M = N / 2;
    constexpr int T = M / E;
    constexpr int S = smem_stride<M, E, false>();
    using TM = Team<M, E, true, sync_kind(T, T * ROWS)>;
    extern __shared__ float2 smem[];
    pdl_wait();
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint64_t row = (uint64_t)blockIdx.x * ROWS + rl;
    const bool ok = row < batch;
    const float2* src = in + row * (M + 1);
    float2* dst = out + row * M;
    float2* sm = smem + rl * S;
    // stage bins 0..M-1 once (coalesced), then pair bin k with bin M-k from shared memory; the
    // Nyquist bin M pairs only with bin 0 and is read directly
    const float2 nyq = (ok && t == 0) ? ld_stream(src + M) : make_float2(0.f, 0.f);   // before the barrier
    float2 v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = ok ? ld_stream(src + t + i * T) : make_float2(0.f, 0.f);   // all loads in flight
#pragma unroll
    for (int i = 0; i < E; ++i) sm[spad(t + i * T)] = v[i];
    TM::sync(rl);
    TM::load_first(v, t, [&](int k) {
        return c2r_split(sm[spad(k)], k == 0 ? nyq : sm[spad(M - k)], k, __ldg(twr + k), s_edge, s_int, out_scale);
    });
    TM::sync(rl);   // the passes reuse the staging buffer for their exchanges
    TM::template passes<0>(v, sm, tw, t, rl);
    pdl_trigger();
    if (ok) TM::for_each_out(v, t, [&](int i, float2 x) { st_stream(dst + i, x); });
}

// ------------------------------------------------------------------ column FFTs
// NY-point FFTs down the columns of a batch of row-major matrices:
//   in[m*matStride + i*pitch + col], i < NY, col < ncols, m < gridDim.x / colBlocks.
// Serves the column pass of a 2-D transform ([batch][ny][nx]: pitch = nx, matStride = ny*nx)
// and transforms along a middle axis of a contiguous [outer][n][inner] array (pitch = inner).
// C consecutive columns per CTA with the column index fastest across threads, so every row
// access is one C*8-byte segment; columns at or past ncols compute on zeros and store nothing.
// Every load precedes the CTA's first __syncthreads and every store follows its last, so
// in == out is allowed.
template <int NY, int E, int C, bool INV>
__global__ void __launch_bounds__((NY / E) * C, min_blocks_64regs((NY / E) * C))
k_cols(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
       uint32_t ncols, uint64_t pitch, uint64_t matStride, uint32_t colBlocks, float scale) {
    constexpr int S = smem_stride<NY, E, true>();
    using TM = Team<NY, E, INV, kSyncBlock>;
    static_assert(TM::P >= 2, "in-place safety needs a barrier between loads and stores");
    extern __shared__ float2 smem[];
    const int c = threadIdx.x % C;
    const int t = threadIdx.x / C;
    const uint64_t m = blockIdx.x / colBlocks;
    const uint32_t col = (blockIdx.x % colBlocks) * C + c;
    const bool live = col < ncols;
    const float2* src = in + m * matStride + (live ? col : 0u);
    float2* dst = out + m * matStride + col;
    float2 v[E];
    TM::run(v, smem + c * S, tw, t, 0, [&](int i) {
        return live ? ld_once_ca(src + (size_t)i * pitch) : make_float2(0.f, 0.f);
    });
    if (live) TM::for_each_out(v, t, [&](int k, float2 x) { st_stream(dst + (size_t)k * pitch, cscale(x, scale)); });
}

// ------------------------------------------------------------------ four-step long C2C
// x[b][N2*n1 + n2] -> (pass A) y[b][N2*k1 + n2] = W_N^(n2*k1) * FFT_N1 over n1
//                  -> (pass B) X[b][k1 + N1*k2]  = FFT_N2 over n2 of y[b][N2*k1 + :]
// W_N^m for m < N is assembled from two FP64-built tables: tlo[m & 255] * thi[m >> 8].

// Pass A: C consecutive columns per CTA, column index fastest across threads so each global
// access is C consecutive complex values (C*8 bytes).
template <int N1, int E, int C, bool INV>
__global__ void __launch_bounds__((N1 / E) * C, 3)
k_long_a(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
         const float2* __restrict__ tlo, const float2* __restrict__ thi, uint64_t batch, int logN2) {
    constexpr int T = N1 / E;
    constexpr int S = smem_stride<N1, E, true>();
    using TM = Team<N1, E, INV, kSyncBlock>;
    extern __shared__ float2 smem[];
    const int c = threadIdx.x % C;
    const int t = threadIdx.x / C;
    const uint32_t N2 = 1u << logN2;
    const uint32_t colBlocks = N2 / C;
    const uint64_t b = blockIdx.x / colBlocks;
    const uint32_t n2 = (blockIdx.x % colBlocks) * C + c;
    const uint64_t N = (uint64_t)N1 << logN2;
    const float2* src = in + b * N + n2;
    float2* dst = out + b * N + n2;
    (void)batch;
    float2 v[E];
    TM::run(v, smem + c * S, tw, t, 0, [&](int i) { return ld_once_ca(src + ((size_t)i << logN2)); });
    TM::for_each_out(v, t, [&](int k1, float2 x) {
        const uint32_t m = n2 * (uint32_t)k1;
        const float2 w = cmul<false>(__ldg(thi + (m >> 8)), __ldg(tlo + (m & 255u)));
        st_stream(dst + ((size_t)k1 << logN2), cmul<INV>(x, w));
    });
}

// Pass B: C consecutive rows per CTA; loads row-contiguous, FFT, then a shared-memory
// transpose so the stride-N1 output is written as C consecutive complex values per k2.
template <int N2, int E, int C, bool INV>
__global__ void __launch_bounds__((N2 / E) * C)
k_long_b(const float2* __restrict__ in, float2* __restrict__ out, const float2* __restrict__ tw,
         uint64_t batch, int logN1, float scale) {
    constexpr int T = N2 / E;
    constexpr int S = smem_stride<N2, E, false>();
    using TM = Team<N2, E, INV, sync_kind(T, T * C)>;
    extern __shared__ float2 smem[];
    const int rl = threadIdx.x / T;
    const int t = threadIdx.x - rl * T;
    const uint32_t N1 = 1u << logN1;
    const uint32_t rowBlocks = N1 / C;
    const uint64_t b = blockIdx.x / rowBlocks;
    const uint32_t k1_0 = (blockIdx.x % rowBlocks) * C;
    const uint64_t N = (uint64_t)N2 << logN1;
    const float2* src = in + b * N + (uint64_t)(k1_0 + rl) * N2;
    float2* sm = smem + rl * S;
    (void)batch;
    float2 v[E];
    TM::run(v, sm, tw, t, rl, [&](int i) { return ld_once_ca(src + i); });
    __syncthreads();
    TM::for_each_out(v, t, [&](int i, float2 x) { sm[spad(i)] = x; });
    __syncthreads();
    float2* dst = out + b * N + k1_0;
    for (int idx = threadIdx.x; idx < C * N2; idx += blockDim.x) {
        const int c = idx % C;
        const int k2 = idx / C;
        st_stream(dst + c + ((size_t)k2 << logN1), cscale(smem[c * S + spad(k2)], scale));
    }
}

// ------------------------------------------------------------------ FP64 twiddle builders
// Stockham table of Sched<N,E>: pass p >= 1 holds exp(-2*pi*i*r*k/(Ns*R)) at
// twoff(p) + (r-1)*Ns + k.  The only FP64 arithmetic in the library.
template <int N, int E>
__global__ void k_tw_stockham(float2* __restrict__ tw) {
    using Sd = Sched<N, E>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Sd::TWSIZE) return;
    int p = 1;
    while (p + 1 < Sd::P && i >= Sd::twoff(p + 1)) ++p;
    const int rel = i - Sd::twoff(p);
    const int ns = Sd::ns(p);
    const int R = Sd::radix(p);
    const int r = rel / ns + 1;
    const int k = rel % ns;
    double s, c;
    sincospi(-2.0 * (double)(r * k) / (double)(ns * R), &s, &c);
    tw[i] = make_float2((float)c, (float)s);
}

// tw[i] = exp(-2*pi*i*(i*stride)/N), i < count.
static __global__ void k_tw_linear(float2* __restrict__ tw, int count, long long stride, long long n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long m = ((long long)i * stride) % n;
    double s, c;
    sincospi(-2.0 * (double)m / (double)n, &s, &c);
    tw[i] = make_float2((float)c, (float)s);
}

}  // namespace dev
}  // namespace bfly
