// Work-list entry of the ragged persistent launch, shared by the host runtime (plan.cpp) and
// the kernel (k_ragged.cu).  Plain-old-data, 64 bytes.
#pragma once
#include <stdint.h>

namespace bfly {

struct RaggedEntry {
    const void* in;      // [batch][n] complex64 rows
    void* out;           // [batch][n] complex64 rows
    const void* tw;      // Stockham twiddle table of (n, 16)
    uint64_t batch;
    uint64_t tile0;      // global index of this request's first tile
    uint32_t logn;       // 5..12
    int32_t direction;   // -1 forward, +1 inverse
    float scale;
    uint32_t rowsPerTile;
    uint64_t reserved;
};
static_assert(sizeof(RaggedEntry) == 64, "RaggedEntry must stay 64 bytes");

// Register radix and CTA size of the ragged kernel: every tile is 256 threads x 16 complex
// values = 4096 points (one 4096-point row, or 4096/n rows of a shorter length).
constexpr int kRaggedE = 16;
constexpr int kRaggedThreads = 256;
constexpr uint32_t kRaggedMinN = 32, kRaggedMaxN = 4096;

}  // namespace bfly
