/* Test infrastructure only.  C restatement of the reference's FP64 CPU oracle
 * (TruNcat3/ascend-fft src/framework/reference.cpp, include/butterfly/reference.hpp):
 *   orc_ref_fft  reference.cpp:14-50  radix-2 DIT in double: bit-reversal gather, twiddle
 *                table w[i] = exp(-2 pi i / n) computed with cos/sin, butterflies
 *                u + w*v / u - w*v, outputs rounded to fp32;
 *   orc_ref_r2c  reference.cpp:55-62  real input as complex, first n/2+1 bins;
 *   orc_ref_c2r  reference.cpp:64-79  mirror X[n-k] = conj X[k] (k = 1..m-1) over bins 0..m
 *                taken as given, y = FFT(conj X) in the fp32 round trip of refFftF32,
 *                out = Re(y)/n in fp32;
 *   orc_max_rel_scaled reference.hpp:30-41, orc_pattern_at reference.cpp:10-12.
 * Pinned against the reference's own compiled oracle (oracle/_ref) by tests/test_oracle.py. */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static uint32_t ilog2(uint32_t n) {
    uint32_t l = 0;
    while ((1u << l) < n) ++l;
    return l;
}

void orc_ref_fft(const float* in, float* out, uint32_t n) {
    if (!n) return;
    double complex* a = malloc(sizeof(double complex) * n);
    double complex* w = malloc(sizeof(double complex) * (n / 2 + 1));
    uint32_t logn = ilog2(n);
    for (uint32_t i = 0; i < n; ++i) {       /* a[i] = x[bitrev(i)] */
        uint32_t r = 0, t = i;
        for (uint32_t b = 0; b < logn; ++b) {
            r = (r << 1) | (t & 1u);
            t >>= 1;
        }
        a[i] = (double)in[2 * r] + I * (double)in[2 * r + 1];
    }
    for (uint32_t i = 0; i < n / 2; ++i) {
        const double ang = -2.0 * M_PI * (double)i / (double)n;
        w[i] = cos(ang) + I * sin(ang);
    }
    for (uint32_t len = 2; len <= n; len <<= 1) {
        const uint32_t half = len >> 1, step = n / len;
        for (uint32_t base = 0; base < n; base += len)
            for (uint32_t j = 0; j < half; ++j) {
                const double complex u = a[base + j];
                const double complex v = a[base + j + half] * w[j * step];
                a[base + j] = u + v;
                a[base + j + half] = u - v;
            }
    }
    for (uint32_t i = 0; i < n; ++i) {
        out[2 * i] = (float)creal(a[i]);
        out[2 * i + 1] = (float)cimag(a[i]);
    }
    free(a);
    free(w);
}

void orc_ref_r2c(const float* in, float* out, uint32_t n) {
    if (n < 2) return;
    float* c = calloc(2 * (size_t)n, sizeof(float));
    float* y = malloc(sizeof(float) * 2 * (size_t)n);
    for (uint32_t j = 0; j < n; ++j) c[2 * j] = in[j];
    orc_ref_fft(c, y, n);
    memcpy(out, y, sizeof(float) * (n + 2));
    free(c);
    free(y);
}

void orc_ref_c2r(const float* in, float* out, uint32_t n) {
    if (n < 2) return;
    const uint32_t m = n >> 1;
    float* c = malloc(sizeof(float) * 2 * (size_t)n);
    float* y = malloc(sizeof(float) * 2 * (size_t)n);
    /* conj of the mirrored full spectrum, each value rounded through float like the reference */
    for (uint32_t k = 0; k <= m; ++k) {
        c[2 * k] = in[2 * k];
        c[2 * k + 1] = -in[2 * k + 1];
    }
    for (uint32_t k = 1; k < m; ++k) {
        c[2 * (n - k)] = in[2 * k];
        c[2 * (n - k) + 1] = in[2 * k + 1];
    }
    orc_ref_fft(c, y, n);
    for (uint32_t j = 0; j < n; ++j) out[j] = y[2 * j] / (float)n;
    free(c);
    free(y);
}

double orc_max_rel_scaled(const float* got, const float* ref, size_t len) {
    if (len && (!got || !ref)) return INFINITY;
    double scale = 0.0, err = 0.0;
    for (size_t i = 0; i < len; ++i) {
        if (!isfinite(got[i]) || !isfinite(ref[i])) return INFINITY;
        const double r = fabs((double)ref[i]);
        const double e = fabs((double)got[i] - (double)ref[i]);
        if (r > scale) scale = r;
        if (e > err) err = e;
    }
    return err / (scale > 1.0 ? scale : 1.0);
}

float orc_pattern_at(size_t i) {
    const uint32_t h = (uint32_t)i * 2654435761u;
    return (float)(h % 1000u) / 1000.f - 0.5f;
}
