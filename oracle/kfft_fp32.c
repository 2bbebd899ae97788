/* Test infrastructure only.  C restatement of the fp32 arithmetic of the reference's AscendC
 * kernels (TruNcat3/ascend-fft), standing in for their device output, which needs an Ascend
 * NPU.  Storage mechanics (UB plane layout, Gather index tables, batch folding) do not change
 * the values and are not restated; the arithmetic and its order are:
 *
 *   twiddle table   butterfly.cpp:96-109 genTwiddles: per stage h a slot of h entries
 *                   exp(-i pi j / h) computed in double and rounded to fp32; negated
 *                   imaginary part for the C2R sign (butterfly.cpp:623).
 *   kfft_fwd        fft_radix2.cpp:51-481: bit-reversed input (DIT); stages h < K = planeKFor(n)
 *                   fused pairwise into radix-4 with W = slot_2h[j2], W^2 = slot_h[j2] and
 *                   W^3 = W*W^2 formed in fp32 (:202-217, :225-247); a residual radix-2 stage
 *                   when log2 K is odd (:316-378); radix-2 stages h >= K in the
 *                   Mul + MulAddDst form re = i1*(-ti) + r1*tr, im = i1*tr + r1*ti (:429-438).
 *                   xflip (C2R) negates the cross rotation s (:190-194).
 *   kfft_r2c_post   fft_real.cpp:47-162: E = (a+conj b)/2, O = (a-conj b)/(2i), t = W_n^k O,
 *                   out[k] = E + t (k <= n/4), out[m-k] = conj(E - t) for the upper half.
 *   kfft_c2r_prep   fft_real.cpp:167-223: bins 0..m as given, bins m..n-1 = conj(X[n-k]).
 *   kfft_c2r_post   fft_real.cpp:228-267: out = Re(y) * (1/n).
 *   planeKFor       include/butterfly/fft_k.hpp:45-85 (vector-op count model).
 *
 * AscendC does not specify whether Axpy / MulAddDst round once (fused) or twice; this
 * restatement rounds every product and every sum separately (compiled with
 * -ffp-contract=off), which is one source of last-ulp differences from the device. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static uint32_t ilog2(uint32_t n) {
    uint32_t l = 0;
    while ((1u << l) < n) ++l;
    return l;
}

/* K-plane factor: smallest vector-op count over K in {kMin..32}, ties to the larger K. */
uint32_t orc_plane_k(uint32_t n) {
    const uint32_t kNeed = (n + 63u) >> 6;
    const uint32_t kMin = (n <= 1024u && kNeed > 8u) ? kNeed : 8u;
    uint32_t best = kMin;
    unsigned long long bestOps = ~0ull;
    const uint32_t logn = ilog2(n);
    for (uint32_t K = kMin; K <= 32u; K <<= 1) {
        if (K * 8u > n) break;
        const uint32_t logK = ilog2(K);
        unsigned long long ops = 0;
        uint32_t si = 0;
        for (; si + 1u < logK; si += 2u) {
            const uint32_t h = 1u << si;
            ops += (unsigned long long)(K / (4u * h)) * (16ull + (unsigned long long)(h - 1u) * 28ull);
        }
        if (si < logK) {
            const uint32_t h = 1u << si;
            const unsigned long long pairs = K / 2u, triv = K / (2u * h);
            ops += triv * 6ull + (pairs - triv) * 8ull;
        }
        for (uint32_t s = logK; s < logn; ++s) {
            const uint32_t h = 1u << s, groups = n / (2u * h), nSlice = (h + 63u) >> 6;
            const int merge = h >= 8u && (2u * h) % 8u == 0u && (2u * h) / 8u <= 255u &&
                              h / 8u <= 255u && groups <= 255u && nSlice <= groups;
            ops += merge ? 8ull * nSlice : 8ull * groups;
            ops += 1ull;
        }
        ops += 7ull;
        if (ops <= bestOps) {
            bestOps = ops;
            best = K;
        }
    }
    return best;
}

/* fp32 helpers with one rounding per operation */
static float fmul(float a, float b) { volatile float r = a * b; return r; }
static float fadd(float a, float b) { volatile float r = a + b; return r; }
static float fsub(float a, float b) { volatile float r = a - b; return r; }

typedef struct { float *re, *im; } planes;

/* slot table for a forward (sign -1) or conjugated (sign +1) transform of length n */
static void twiddles(uint32_t n, int sign, float** twr, float** twi, uint32_t** slotOf) {
    const uint32_t logn = ilog2(n);
    *twr = calloc(n + 16u, sizeof(float));
    *twi = calloc(n + 16u, sizeof(float));
    *slotOf = calloc(logn + 1u, sizeof(uint32_t));
    uint32_t off = 0, s = 0;
    for (uint32_t h = 1; h <= n / 2u; h <<= 1, ++s) {
        (*slotOf)[s] = off;
        for (uint32_t j = 0; j < h; ++j) {
            const double ang = -M_PI * (double)j / (double)h;
            (*twr)[off + j] = (float)cos(ang);
            (*twi)[off + j] = (float)sin(ang);
            if (sign > 0) (*twi)[off + j] = -(*twi)[off + j];
        }
        off += (h + 7u) & ~7u;
    }
}

void orc_kfft_fwd(const float* in, float* out, uint32_t n, int sign) {
    const uint32_t logn = ilog2(n), K = orc_plane_k(n), logK = ilog2(K);
    const int xflip = sign > 0;
    float *twr, *twi;
    uint32_t* slot;
    twiddles(n, sign, &twr, &twi, &slot);
    planes a = {malloc(sizeof(float) * n), malloc(sizeof(float) * n)};
    for (uint32_t i = 0; i < n; ++i) {   /* DIT: bit-reversed gather */
        uint32_t r = 0, t = i;
        for (uint32_t b = 0; b < logn; ++b) {
            r = (r << 1) | (t & 1u);
            t >>= 1;
        }
        a.re[i] = in[2 * r];
        a.im[i] = in[2 * r + 1];
    }
    uint32_t si = 0;
    /* plane region: stage pairs (h, 2h) as radix-4 */
    for (; si + 1u < logK; si += 2u) {
        const uint32_t h = 1u << si;
        const uint32_t sW2 = slot[si], sW = slot[si + 1];
        for (uint32_t b0 = 0; b0 < n; b0 += 4u * h)
            for (uint32_t j2 = 0; j2 < h; ++j2) {
                const uint32_t i0 = b0 + j2, i1 = i0 + h, i2 = i0 + 2u * h, i3 = i0 + 3u * h;
                float r0 = a.re[i0], c0 = a.im[i0], r1 = a.re[i1], c1 = a.im[i1];
                float r2 = a.re[i2], c2 = a.im[i2], r3 = a.re[i3], c3 = a.im[i3];
                float u0, u1, u2, u3, u4, u5;
                if (j2 != 0) {
                    const float w2r = twr[sW2 + j2], w2i = twi[sW2 + j2];
                    const float wr = twr[sW + j2], wi = twi[sW + j2];
                    const float w3r = fsub(fmul(wr, w2r), fmul(wi, w2i));
                    const float w3i = fadd(fmul(wr, w2i), fmul(wi, w2r));
                    u0 = fadd(fmul(r1, w2r), fmul(c1, -w2i));
                    u1 = fadd(fmul(r1, w2i), fmul(c1, w2r));
                    u2 = fadd(fmul(r2, wr), fmul(c2, -wi));
                    u3 = fadd(fmul(r2, wi), fmul(c2, wr));
                    u4 = fadd(fmul(r3, w3r), fmul(c3, -w3i));
                    u5 = fadd(fmul(r3, w3i), fmul(c3, w3r));
                } else {
                    u0 = r1; u1 = c1; u2 = r2; u3 = c2; u4 = r3; u5 = c3;
                }
                const float qr = fsub(r0, u0), qi = fsub(c0, u1);
                const float pr = fadd(r0, u0), pi = fadd(c0, u1);
                const float sr = xflip ? fsub(u4, u2) : fsub(u2, u4);
                const float sI = xflip ? fsub(u5, u3) : fsub(u3, u5);
                const float rr = fadd(u2, u4), ri = fadd(u3, u5);
                a.re[i2] = fsub(pr, rr); a.im[i2] = fsub(pi, ri);
                a.re[i0] = fadd(pr, rr); a.im[i0] = fadd(pi, ri);
                a.re[i3] = fsub(qr, sI); a.im[i3] = fadd(qi, sr);
                a.re[i1] = fadd(qr, sI); a.im[i1] = fsub(qi, sr);
            }
    }
    /* remaining stages: radix-2 (the residual plane stage, then the planar stages) */
    for (uint32_t s = si; s < logn; ++s) {
        const uint32_t h = 1u << s, sl = slot[s];
        const int planar = s >= logK;
        for (uint32_t b0 = 0; b0 < n; b0 += 2u * h)
            for (uint32_t j = 0; j < h; ++j) {
                const uint32_t p = b0 + j, q = p + h;
                const float tr = twr[sl + j], ti = twi[sl + j];
                float xr, xi;
                if (planar) {   /* Mul + MulAddDst */
                    xr = fadd(fmul(a.re[q], tr), fmul(a.im[q], -ti));
                    xi = fadd(fmul(a.re[q], ti), fmul(a.im[q], tr));
                } else if (tr == 1.0f && ti == 0.0f) {
                    xr = a.re[q];
                    xi = a.im[q];
                } else {        /* Muls + Axpy */
                    xr = fadd(fmul(a.re[q], tr), fmul(a.im[q], -ti));
                    xi = fadd(fmul(a.re[q], ti), fmul(a.im[q], tr));
                }
                a.re[q] = fsub(a.re[p], xr);
                a.re[p] = fadd(a.re[p], xr);
                a.im[q] = fsub(a.im[p], xi);
                a.im[p] = fadd(a.im[p], xi);
            }
    }
    for (uint32_t i = 0; i < n; ++i) {
        out[2 * i] = a.re[i];
        out[2 * i + 1] = a.im[i];
    }
    free(a.re);
    free(a.im);
    free(twr);
    free(twi);
    free(slot);
}

void orc_kfft_r2c(const float* in, float* out, uint32_t n) {
    const uint32_t m = n >> 1, kmax = n >> 2;
    float* z = malloc(sizeof(float) * n);
    orc_kfft_fwd(in, z, m, -1);   /* real row reused as m interleaved complex values */
    for (uint32_t s = 0; s <= m; ++s) {
        const int lower = s <= kmax;
        const uint32_t idx = lower ? s : m - s;
        const uint32_t bb = idx == 0 ? 0 : m - idx;
        const float ar = z[2 * idx], ai = z[2 * idx + 1], br = z[2 * bb], bi = z[2 * bb + 1];
        const double ang = -2.0 * M_PI * (double)idx / (double)n;
        const float wr = (float)cos(ang), wi = (float)sin(ang);
        const float er = fmul(fadd(ar, br), 0.5f), ei = fmul(fsub(ai, bi), 0.5f);
        const float orr = fmul(fadd(ai, bi), 0.5f), oi = fmul(fsub(br, ar), 0.5f);
        const float tre = fsub(fmul(wr, orr), fmul(wi, oi));
        const float tim = fadd(fmul(wr, oi), fmul(wi, orr));
        out[2 * s] = lower ? fadd(er, tre) : fsub(er, tre);
        out[2 * s + 1] = lower ? fadd(ei, tim) : fsub(tim, ei);
    }
    free(z);
}

void orc_kfft_c2r(const float* in, float* out, uint32_t n) {
    const uint32_t m = n >> 1;
    float* full = malloc(sizeof(float) * 2 * (size_t)n);
    float* y = malloc(sizeof(float) * 2 * (size_t)n);
    for (uint32_t k = 0; k < m; ++k) {            /* bins 0..m-1 as given */
        full[2 * k] = in[2 * k];
        full[2 * k + 1] = in[2 * k + 1];
    }
    for (uint32_t t = 0; t < m; ++t) {            /* bin m+t = conj(bin m-t) */
        full[2 * (m + t)] = in[2 * (m - t)];
        full[2 * (m + t) + 1] = -in[2 * (m - t) + 1];
    }
    orc_kfft_fwd(full, y, n, +1);
    const float sc = 1.0f / (float)n;
    for (uint32_t j = 0; j < n; ++j) out[j] = fmul(y[2 * j], sc);
    free(full);
    free(y);
}
