// Table of compiled kernel variants.  Each kernel translation unit instantiates its templates
// and exposes a lookup; backend_cuda.cu resolves (kind, n, e, cta) to a function pointer plus
// launch geometry.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bfly {
namespace dev {

using KC2C = void (*)(const float2*, float2*, const float2*, uint64_t, float);
using KR2C = void (*)(const float2*, float2*, const float2*, const float2*, uint64_t, float, float);
using KC2R = void (*)(const float2*, float2*, const float2*, const float2*, uint64_t, float,
                      float, float);
using KLongA = void (*)(const float2*, float2*, const float2*, const float2*, const float2*,
                        uint64_t, int);
using KLongB = void (*)(const float2*, float2*, const float2*, uint64_t, int, float);
using KCols = void (*)(const float2*, float2*, const float2*, uint32_t, uint64_t, uint64_t, uint32_t, float);
using KTw = void (*)(float2*);

struct Entry {
    uint32_t n;      // transform length (real length for R2C/C2R)
    int e;           // complex values per thread
    int cta;         // threads per CTA
    int flag;        // C2C: inverse; R2C: weighted; long: inverse
    const void* fn;  // kernel
    int rows;        // transforms per CTA
    int smem;        // dynamic shared memory bytes
};

// Returns nullptr when the variant is not compiled.
const Entry* findC2CFwd(uint32_t n, int e, int cta);
const Entry* findC2CInv(uint32_t n, int e, int cta);
const Entry* findR2C(uint32_t n, int e, int cta, bool weighted);
const Entry* findC2R(uint32_t n, int e, int cta);
const Entry* findLongA(uint32_t n1, bool inverse);
const Entry* findLongB(uint32_t n2, bool inverse);
const Entry* findCols(uint32_t ny, bool inverse);   // rows = columns per CTA
// Stockham twiddle builder for Sched<n,e> and its table size.
bool findTw(uint32_t n, int e, KTw* fn, int* count);

}  // namespace dev
}  // namespace bfly

// Geometry helpers for the instantiation macros.
#define BFLY_ROWS(N, E, CTA) ((CTA) / ((N) / (E)))
