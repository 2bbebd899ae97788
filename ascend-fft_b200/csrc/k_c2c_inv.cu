// C2C kernel instantiations (inverse).  Variant list: N in 32..16384, E in {8,16},
// CTA in {128,256,512} (1024 only for one-transform-per-CTA lengths), shared memory <= 227 KB.
#include "fft_kernels.cuh"
#include "registry.cuh"

namespace bfly {
namespace dev {

#define E_(N, E, CTA) {N, E, CTA, 1, (const void*)&k_c2c<N, E, BFLY_ROWS(N, E, CTA), true>, \
    BFLY_ROWS(N, E, CTA), BFLY_ROWS(N, E, CTA) * smem_stride<N, E, false>() * 8}
static const Entry kTable[] = {
    E_(32, 8, 128),
    E_(32, 8, 256),
    E_(32, 8, 512),
    E_(32, 16, 128),
    E_(32, 16, 256),
    E_(32, 16, 512),
    E_(64, 8, 128),
    E_(64, 8, 256),
    E_(64, 8, 512),
    E_(64, 16, 128),
    E_(64, 16, 256),
    E_(64, 16, 512),
    E_(128, 8, 128),
    E_(128, 8, 256),
    E_(128, 8, 512),
    E_(128, 16, 128),
    E_(128, 16, 256),
    E_(128, 16, 512),
    E_(256, 8, 128),
    E_(256, 8, 256),
    E_(256, 8, 512),
    E_(256, 16, 128),
    E_(256, 16, 256),
    E_(256, 16, 512),
    E_(512, 8, 128),
    E_(512, 8, 256),
    E_(512, 8, 512),
    E_(512, 16, 128),
    E_(512, 16, 256),
    E_(512, 16, 512),
    E_(1024, 8, 128),
    E_(1024, 8, 256),
    E_(1024, 8, 512),
    E_(1024, 16, 128),
    E_(1024, 16, 256),
    E_(1024, 16, 512),
    E_(2048, 8, 256),
    E_(2048, 8, 512),
    E_(2048, 16, 128),
    E_(2048, 16, 256),
    E_(2048, 16, 512),
    E_(4096, 8, 512),
    E_(4096, 16, 256),
    E_(4096, 16, 512),
    E_(8192, 8, 1024),
    E_(8192, 16, 512),
    E_(16384, 16, 1024),
};
#undef E_

const Entry* findC2CInv(uint32_t n, int e, int cta) {
    for (const Entry& x : kTable)
        if (x.n == n && x.e == e && x.cta == cta) return &x;
    return nullptr;
}

}  // namespace dev
}  // namespace bfly
