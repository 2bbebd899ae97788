// FP64 acceptance reference used by Plan::measure / Context::select to accept or reject a
// measured candidate, with the semantics of the reference's acceptance helpers
// (include/butterfly/reference.hpp:14-60, src/framework/reference.cpp:10-79):
//   refFftF32  forward C2C of n interleaved fp32 values computed in double, rounded to fp32;
//   refR2CF32  numpy.fft.rfft layout [n+2];  refC2RF32  numpy.fft.irfft incl. 1/n, DC and
//   Nyquist imaginary parts ignored;  maxRelScaled  max|got-ref| / max(1, max|ref|).
// This checker never produces a transform result for the caller; the device kernels do.
#include "bfly/plan.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <vector>

namespace bfly {

namespace {
using cd = std::complex<double>;

// In-place iterative radix-2 transform in double precision (sign -1 forward).
void fftDouble(std::vector<cd>& a, int sign) {
    const size_t n = a.size();
    if (n < 2) return;
    for (size_t i = 1, j = 0; i < n; ++i) {   // bit-reversal permutation
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j |= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len / 2;
        for (size_t k = 0; k < half; ++k) {
            const double ang = sign * 2.0 * M_PI * (double)k / (double)len;
            const cd w(std::cos(ang), std::sin(ang));
            for (size_t base = 0; base < n; base += len) {
                const cd u = a[base + k];
                const cd v = a[base + k + half] * w;
                a[base + k] = u + v;
                a[base + k + half] = u - v;
            }
        }
    }
}
}  // namespace

void refFftF32(const float* in, float* out, uint32_t n) {
    if (!n) return;
    std::vector<cd> a(n);
    for (uint32_t i = 0; i < n; ++i) a[i] = cd(in[2 * i], in[2 * i + 1]);
    fftDouble(a, -1);
    for (uint32_t i = 0; i < n; ++i) {
        out[2 * i] = (float)a[i].real();
        out[2 * i + 1] = (float)a[i].imag();
    }
}

void refR2CF32(const float* in, float* out, uint32_t n) {
    if (n < 2) return;
    std::vector<cd> a(n);
    for (uint32_t i = 0; i < n; ++i) a[i] = cd(in[i], 0.0);
    fftDouble(a, -1);
    for (uint32_t k = 0; k <= n / 2; ++k) {
        out[2 * k] = (float)a[k].real();
        out[2 * k + 1] = (float)a[k].imag();
    }
}

void refC2RF32(const float* in, float* out, uint32_t n) {
    if (n < 2) return;
    const uint32_t m = n / 2;
    std::vector<cd> a(n);
    a[0] = cd(in[0], 0.0);
    a[m] = cd(in[2 * m], 0.0);
    for (uint32_t k = 1; k < m; ++k) {
        a[k] = cd(in[2 * k], in[2 * k + 1]);
        a[n - k] = std::conj(a[k]);
    }
    fftDouble(a, +1);
    for (uint32_t i = 0; i < n; ++i) out[i] = (float)(a[i].real() / (double)n);
}

double maxRelScaled(const float* got, const float* ref, size_t len) {
    if (len && (!got || !ref)) return std::numeric_limits<double>::infinity();
    double scale = 0.0, err = 0.0;
    for (size_t i = 0; i < len; ++i) {
        if (!std::isfinite(got[i]) || !std::isfinite(ref[i]))
            return std::numeric_limits<double>::infinity();
        scale = std::max(scale, std::fabs((double)ref[i]));
        err = std::max(err, std::fabs((double)got[i] - (double)ref[i]));
    }
    return err / std::max(1.0, scale);
}

// Deterministic test pattern shared with the harnesses: ((i*2654435761) mod 1000)/1000 - 0.5,
// computed in 32-bit unsigned arithmetic like the reference (reference.cpp:10-12).
float patternAt(size_t i) {
    const uint32_t h = (uint32_t)((uint32_t)i * 2654435761u);
    return (float)(h % 1000u) / 1000.f - 0.5f;
}

uint32_t sampleBatches(uint32_t batch, uint32_t want, uint32_t* out, uint32_t maxOut) {
    if (want > maxOut) want = maxOut;
    if (batch == 0 || want == 0) return 0;
    if (batch <= want) {
        for (uint32_t i = 0; i < batch; ++i) out[i] = i;
        return batch;
    }
    if (want == 1) {
        out[0] = 0;
        return 1;
    }
    for (uint32_t i = 0; i < want; ++i)
        out[i] = (uint32_t)((uint64_t)i * (batch - 1) / (want - 1));
    return want;
}

}  // namespace bfly
