// Small odd-length DFTs in registers (3, 5, 7), natural order in and out, forward sign
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

template <bool INV> struct DFT<3, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft3<INV>(v[0], v[1], v[2]); }
};
template <bool INV> struct DFT<5, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft5<INV>(v[0], v[1], v[2], v[3], v[4]); }
};
template <bool INV> struct DFT<7, INV> {
    static __device__ __forceinline__ void run(float2* v) { dft7<INV>(v); }
};

}  // namespace dev
}  // namespace bfly
