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
    uint32_t e;          // complex values per thread (register radix) of this request's tiles
    uint32_t reserved;
};
static_assert(sizeof(RaggedEntry) == 64, "RaggedEntry must stay 64 bytes");

#ifdef __CUDACC__
#define BFLY_HD __host__ __device__
#else
#define BFLY_HD
#endif

// CTA size of the ragged kernel and the register radix per length: a tile is 256 threads x E
// complex values (4096 points for E = 16: one 4096-point row, or 4096/n rows of a shorter
// length; 2048 points for E = 8).  Every length 32..2048 has both variants, 4096 only E = 16
// (256 threads x 8 values cannot hold a row).  raggedE is the default per length (the short
// lengths ran faster with E = 8); the autotuner may choose the other variant per length.
constexpr int kRaggedThreads = 256;
constexpr uint32_t kRaggedMinN = 32, kRaggedMaxN = 4096;
constexpr int kRaggedMinLog = 5, kRaggedMaxLog = 12;
BFLY_HD constexpr int raggedE(int logn) { return logn <= 6 ? 8 : 16; }
BFLY_HD constexpr bool raggedVariant(int logn, int e) {
    return logn >= kRaggedMinLog && logn <= kRaggedMaxLog && (e == 16 || (e == 8 && logn <= 11));
}
BFLY_HD constexpr uint32_t raggedRows(int logn, int e) {
    return (uint32_t)kRaggedThreads / ((1u << logn) / (uint32_t)e);
}
BFLY_HD constexpr uint32_t raggedRows(int logn) { return raggedRows(logn, raggedE(logn)); }
// Default choice as a mask over lengths: bit (log2 n - 5) set = E 8 for that length.
constexpr uint32_t kRaggedDefaultRadix8 = (1u << (6 - kRaggedMinLog + 1)) - 1u;   // n = 32, 64

}  // namespace bfly
