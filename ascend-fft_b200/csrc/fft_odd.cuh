// Small odd-length DFTs in registers (3, 5, 7, 9, 11, 13) and Good-Thomas composites (6, 10,
// 12, 14, 15), natural order in and out, forward sign
// exp(-2*pi*i*j*k/R) (INV flips it), and their DFT<R, INV> specialisations for the radix
// passes.  Each pairs x[m] with x[R-m]: t = x[m] + x[R-m], d = x[m] - x[R-m], then
//   X[k]   = x0 + sum_m cos(2 pi k m / R) t_m  -/+  i sum_m sin(2 pi k m / R) d_m
//   X[R-k] = the same with the sign of the sine part flipped.
// The constants are cos / sin of 2*pi*m/R, rounded to float.
#pragma once
#include "fft_core.cuh"

namespace bfly {
namespace dev {

__device__ __forceinline__ float2 mul_i(float2 a, bool neg) {   // -i*a (neg) or +i*a
    return neg ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

template <bool INV>
__device__ __forceinline__ void dft3(float2& x0, float2& x1, float2& x2) {
    constexpr float kS3 = 0.866025403784438647f;   // sin(2*pi/3)
    const float2 t1 = cadd(x1, x2);
    const float2 t2 = make_float2(x1.x - x2.x, x1.y - x2.y);
    const float2 m = make_float2(x0.x - 0.5f * t1.x, x0.y - 0.5f * t1.y);
    const float2 r = mul_i(make_float2(kS3 * t2.x, kS3 * t2.y), !INV);
    x0 = cadd(x0, t1);
    x1 = cadd(m, r);
    x2 = make_float2(m.x - r.x, m.y - r.y);
}

template <bool INV>
__device__ __forceinline__ void dft5(float2& x0, float2& x1, float2& x2, float2& x3, float2& x4) {
    constexpr float kC1 = 0.309016994374947424f, kC2 = -0.809016994374947424f;   // cos(2pi/5), cos(4pi/5)
    constexpr float kS1 = 0.951056516295153572f, kS2 = 0.587785252292473129f;    // sin(2pi/5), sin(4pi/5)
    const float2 t1 = cadd(x1, x4), t2 = cadd(x2, x3);
    const float2 t3 = make_float2(x1.x - x4.x, x1.y - x4.y), t4 = make_float2(x2.x - x3.x, x2.y - x3.y);
    const float2 a1 = make_float2(x0.x + kC1 * t1.x + kC2 * t2.x, x0.y + kC1 * t1.y + kC2 * t2.y);
    const float2 a2 = make_float2(x0.x + kC2 * t1.x + kC1 * t2.x, x0.y + kC2 * t1.y + kC1 * t2.y);
    const float2 b1 = mul_i(make_float2(kS1 * t3.x + kS2 * t4.x, kS1 * t3.y + kS2 * t4.y), !INV);
    const float2 b2 = mul_i(make_float2(kS2 * t3.x - kS1 * t4.x, kS2 * t3.y - kS1 * t4.y), !INV);
    x0 = cadd(x0, cadd(t1, t2));
    x1 = cadd(a1, b1);
    x4 = make_float2(a1.x - b1.x, a1.y - b1.y);
    x2 = cadd(a2, b2);
    x3 = make_float2(a2.x - b2.x, a2.y - b2.y);
}

template <bool INV>
__device__ __forceinline__ void dft7(float2* x) {
    constexpr float kC1 = 0.623489801858733531f, kC2 = -0.222520933956314404f, kC3 = -0.900968867902419126f;
    constexpr float kS1 = 0.781831482468029809f, kS2 = 0.974927912181823607f, kS3 = 0.433883739117558120f;
    const float2 t1 = cadd(x[1], x[6]), t2 = cadd(x[2], x[5]), t3 = cadd(x[3], x[4]);
    const float2 d1 = csub(x[1], x[6]), d2 = csub(x[2], x[5]), d3 = csub(x[3], x[4]);
    const float2 x0 = x[0];
    // cos(2 pi k m / 7) and sin(2 pi k m / 7) for k, m in 1..3 reduce to +-C1..C3, +-S1..S3
    const float2 a1 = make_float2(x0.x + kC1 * t1.x + kC2 * t2.x + kC3 * t3.x, x0.y + kC1 * t1.y + kC2 * t2.y + kC3 * t3.y);
    const float2 a2 = make_float2(x0.x + kC2 * t1.x + kC3 * t2.x + kC1 * t3.x, x0.y + kC2 * t1.y + kC3 * t2.y + kC1 * t3.y);
    const float2 a3 = make_float2(x0.x + kC3 * t1.x + kC1 * t2.x + kC2 * t3.x, x0.y + kC3 * t1.y + kC1 * t2.y + kC2 * t3.y);
    const float2 b1 = mul_i(make_float2(kS1 * d1.x + kS2 * d2.x + kS3 * d3.x, kS1 * d1.y + kS2 * d2.y + kS3 * d3.y), !INV);
    const float2 b2 = mul_i(make_float2(kS2 * d1.x - kS3 * d2.x - kS1 * d3.x, kS2 * d1.y - kS3 * d2.y - kS1 * d3.y), !INV);
    const float2 b3 = mul_i(make_float2(kS3 * d1.x - kS1 * d2.x + kS2 * d3.x, kS3 * d1.y - kS1 * d2.y + kS2 * d3.y), !INV);
    x[0] = cadd(x0, cadd(t1, cadd(t2, t3)));
    x[1] = cadd(a1, b1);
    x[6] = csub(a1, b1);
    x[2] = cadd(a2, b2);
    x[5] = csub(a2, b2);
    x[3] = cadd(a3, b3);
    x[4] = csub(a3, b3);
}

// Odd prime R = 11, 13 by the same symmetric pairs: (R-1)/2 cosine and sine sums per output pair.
// cos / sin of 2 pi q / R for q = 1 .. (R-1)/2; larger q by symmetry (cos even, sin odd about R/2).
__host__ __device__ constexpr float cos11(int q) {
    switch (q) {
        case 1: return 8.412535328311812055e-1f;
        case 2: return 4.154150130018864351e-1f;
        case 3: return -1.423148382732851436e-1f;
        case 4: return -6.548607339452851006e-1f;
        case 5: return -9.594929736144973687e-1f;
        default: return 0.f;
    }
}
__host__ __device__ constexpr float sin11(int q) {
    switch (q) {
        case 1: return 5.406408174555975554e-1f;
        case 2: return 9.096319953545183301e-1f;
        case 3: return 9.898214418809326842e-1f;
        case 4: return 7.557495743542582689e-1f;
        case 5: return 2.817325568414296710e-1f;
        default: return 0.f;
    }
}
__host__ __device__ constexpr float cos13(int q) {
    switch (q) {
        case 1: return 8.854560256532099105e-1f;
        case 2: return 5.680647467311558119e-1f;
        case 3: return 1.205366802553230476e-1f;
        case 4: return -3.546048870425356214e-1f;
        case 5: return -7.485107481711010813e-1f;
        case 6: return -9.709418174260520118e-1f;
        default: return 0.f;
    }
}
__host__ __device__ constexpr float sin13(int q) {
    switch (q) {
        case 1: return 4.647231720437685620e-1f;
        case 2: return 8.229838658936563522e-1f;
        case 3: return 9.927088740980539727e-1f;
        case 4: return 9.350162426854148334e-1f;
        case 5: return 6.631226582407951931e-1f;
        case 6: return 2.393156642875577667e-1f;
        default: return 0.f;
    }
}
template <int R>
__host__ __device__ constexpr float prime_cos(int q) {
    const int r = q <= R / 2 ? q : R - q;
    return q == 0 ? 1.f : (R == 11 ? cos11(r) : cos13(r));
}
template <int R>
__host__ __device__ constexpr float prime_sin(int q) {
    const int r = q <= R / 2 ? q : R - q;
    const float v = R == 11 ? sin11(r) : sin13(r);
    return q <= R / 2 ? v : -v;
}

template <int R, bool INV>
__device__ __forceinline__ void dft_prime(float2* x) {
    constexpr int H = (R - 1) / 2;
    float2 t[H + 1], d[H + 1];
#pragma unroll
    for (int m = 1; m <= H; ++m) {
        t[m] = cadd(x[m], x[R - m]);
        d[m] = csub(x[m], x[R - m]);
    }
    const float2 x0 = x[0];
    float2 sum = x0;
#pragma unroll
    for (int m = 1; m <= H; ++m) sum = cadd(sum, t[m]);
#pragma unroll
    for (int k = 1; k <= H; ++k) {
        float2 a = x0, b = make_float2(0.f, 0.f);
#pragma unroll
        for (int m = 1; m <= H; ++m) {
            const float c = prime_cos<R>((k * m) % R), s = prime_sin<R>((k * m) % R);
            a = make_float2(fmaf(c, t[m].x, a.x), fmaf(c, t[m].y, a.y));
            b = make_float2(fmaf(s, d[m].x, b.x), fmaf(s, d[m].y, b.y));
        }
        b = mul_i(b, !INV);
        x[k] = cadd(a, b);
        x[R - k] = csub(a, b);
    }
    x[0] = sum;
}

// 9 = 3 x 3 Cooley-Tukey: j = 3 j1 + j2, k = k1 + 3 k2, inner twiddles W_9^(j2 k1).
template <bool INV>
__device__ __forceinline__ void dft9(float2* v) {
    constexpr float kC1 = 0.766044443118978035f, kS1 = 0.642787609686539326f;    // 2pi/9
    constexpr float kC2 = 0.173648177666930349f, kS2 = 0.984807753012208060f;    // 4pi/9
    constexpr float kC4 = -0.939692620785908384f, kS4 = 0.342020143325668734f;   // 8pi/9
#pragma unroll
    for (int j2 = 0; j2 < 3; ++j2) dft3<INV>(v[j2], v[3 + j2], v[6 + j2]);   // v[3 k1 + j2]
    const float2 w1 = make_float2(kC1, -kS1), w2 = make_float2(kC2, -kS2), w4 = make_float2(kC4, -kS4);
    v[4] = cmul<INV>(v[4], w1);   // k1 = 1, j2 = 1
    v[5] = cmul<INV>(v[5], w2);   // k1 = 1, j2 = 2
    v[7] = cmul<INV>(v[7], w2);   // k1 = 2, j2 = 1
    v[8] = cmul<INV>(v[8], w4);   // k1 = 2, j2 = 2
    float2 y[9];
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
        float2 a = v[3 * k1], b = v[3 * k1 + 1], c = v[3 * k1 + 2];
        dft3<INV>(a, b, c);
        y[k1] = a;
        y[k1 + 3] = b;
        y[k1 + 6] = c;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) v[k] = y[k];
}

// x with (a * x) mod m == 1 (gcd(a, m) = 1; 0 for m = 1), at compile time.
__host__ __device__ constexpr int mod_inv(int a, int m) {
    for (int x = 1; x < m; ++x)
        if ((a * x) % m == 1) return x;
    return 0;
}

template <int R, bool INV> struct DFT;

// R = A*B with gcd(A, B) = 1 by Good-Thomas, no inner twiddles: input j = CRT(j1, j2)
// (j = j1 mod A, j = j2 mod B), output k = (B k1 + A k2) mod R.
template <int A, int B, bool INV>
__device__ __forceinline__ void dft_pfa(float2* v) {
    constexpr int R = A * B;
    constexpr int U = B * mod_inv(B % A, A), V = A * mod_inv(A % B, B);
    float2 y[R];   // y[j1 B + k2]
#pragma unroll
    for (int j1 = 0; j1 < A; ++j1) {
        float2 c[B];
#pragma unroll
        for (int j2 = 0; j2 < B; ++j2) c[j2] = v[(j1 * U + j2 * V) % R];
        DFT<B, INV>::run(c);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) y[j1 * B + k2] = c[k2];
    }
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) {
        float2 c[A];
#pragma unroll
        for (int j1 = 0; j1 < A; ++j1) c[j1] = y[j1 * B + k2];
        DFT<A, INV>::run(c);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) v[(B * k1 + A * k2) % R] = c[k1];
    }
}

template <bool INV> struct DFT<3, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft3<INV>(v[0], v[1], v[2]); }
};
template <bool INV> struct DFT<5, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft5<INV>(v[0], v[1], v[2], v[3], v[4]); }
};
template <bool INV> struct DFT<7, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft7<INV>(v); }
};
template <bool INV> struct DFT<11, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_prime<11, INV>(v); }
};
template <bool INV> struct DFT<13, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_prime<13, INV>(v); }
};
template <bool INV> struct DFT<9, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft9<INV>(v); }
};
template <bool INV> struct DFT<6, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_pfa<2, 3, INV>(v); }
};
template <bool INV> struct DFT<10, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_pfa<2, 5, INV>(v); }
};
template <bool INV> struct DFT<12, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_pfa<4, 3, INV>(v); }
};
template <bool INV> struct DFT<14, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_pfa<2, 7, INV>(v); }
};
template <bool INV> struct DFT<15, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft_pfa<3, 5, INV>(v); }
};

}  // namespace dev
}  // namespace bfly
