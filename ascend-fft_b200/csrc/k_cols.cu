// Column-FFT instantiations (k_cols): NY in 32..4096, radix 16.  Columns per CTA (C) set the
// width of every row segment a CTA reads and writes (C*8 bytes); narrow segments scatter
// across DRAM pages, so C is as large as one CTA's shared memory (C*NY*8 bytes + padding)
// allows: 128-byte segments up to NY = 1024, 64 at 2048, 32 at 4096.
#include "fft_kernels.cuh"
#include "registry.cuh"

namespace bfly {
namespace dev {

#define KC_(NY, C, INV) {NY, 16, (NY / 16) * C, INV, (const void*)&k_cols<NY, 16, C, INV>, C, \
    C * smem_stride<NY, 16, true>() * 8}
static const Entry kCols[] = {
    KC_(32, 128, false), KC_(64, 64, false), KC_(128, 32, false), KC_(256, 16, false),
    KC_(512, 16, false), KC_(1024, 16, false), KC_(2048, 8, false), KC_(4096, 4, false),
    KC_(32, 128, true),  KC_(64, 64, true),  KC_(128, 32, true),  KC_(256, 16, true),
    KC_(512, 16, true),  KC_(1024, 16, true),  KC_(2048, 8, true),  KC_(4096, 4, true),
};
#undef KC_

const Entry* findCols(uint32_t ny, bool inverse) {
    for (const Entry& x : kCols)
        if (x.n == ny && x.flag == (int)inverse) return &x;
    return nullptr;
}

}  // namespace dev
}  // namespace bfly
