// extern "C" entry points over the reference's own FP64 oracle, compiled from the reference
// sources in place (src/framework/reference.cpp, include/butterfly/reference.hpp of
// TruNcat3/ascend-fft) into oracle/_ref/libref.so by oracle/Makefile.  Test infrastructure
// only: used to pin the restatements and as the timed CPU reference arm of bench.py.
#include "butterfly/reference.hpp"

#include <cstddef>
#include <cstdint>

extern "C" {

// Forward C2C of `rows` rows [rows][2n] (bfly::refFftF32 per row).
void ref_fft_rows(const float* in, float* out, uint32_t n, uint32_t rows) {
    for (uint32_t r = 0; r < rows; ++r)
        bfly::refFftF32(in + (size_t)r * 2 * n, out + (size_t)r * 2 * n, n);
}

// R2C rows [rows][n] -> [rows][n+2] (bfly::refR2CF32).
void ref_r2c_rows(const float* in, float* out, uint32_t n, uint32_t rows) {
    for (uint32_t r = 0; r < rows; ++r)
        bfly::refR2CF32(in + (size_t)r * n, out + (size_t)r * (n + 2), n);
}

// C2R rows [rows][n+2] -> [rows][n] (bfly::refC2RF32).
void ref_c2r_rows(const float* in, float* out, uint32_t n, uint32_t rows) {
    for (uint32_t r = 0; r < rows; ++r)
        bfly::refC2RF32(in + (size_t)r * (n + 2), out + (size_t)r * n, n);
}

double ref_max_rel_scaled(const float* got, const float* ref, size_t len) {
    return bfly::maxRelScaled(got, ref, len);
}

float ref_pattern_at(size_t i) { return bfly::patternAt(i); }

uint32_t ref_sample_batches(uint32_t batch, uint32_t want, uint32_t* out, uint32_t max_out) {
    return bfly::sampleBatches(batch, want, out, max_out);
}

}  // extern "C"
