// Four-step long C2C instantiations.  N = N1 * 256 with N1 in {32, 64, 128, 256}
// (N = 8192 .. 65536), register radix 16 in both passes, 256-thread CTAs:
//   pass A: N1-point column FFTs, C = 256 / (N1/16) columns per CTA;
//   pass B: 256-point row FFTs, 16 rows per CTA.
// Also the Stockham twiddle-builder table for every (N, E) the library instantiates.
#include "fft_kernels.cuh"
#include "registry.cuh"

namespace bfly {
namespace dev {

#define LA_(N1, INV) {N1, 16, 256, INV, (const void*)&k_long_a<N1, 16, 256 / (N1 / 16), INV>, \
    256 / (N1 / 16), (256 / (N1 / 16)) * smem_stride<N1, 16, true>() * 8}
#define LB_(N2, INV) {N2, 16, 256, INV, (const void*)&k_long_b<N2, 16, 256 / (N2 / 16), INV>, \
    256 / (N2 / 16), (256 / (N2 / 16)) * smem_stride<N2, 16, false>() * 8}
static const Entry kLongA[] = {
    LA_(32, false), LA_(64, false), LA_(128, false), LA_(256, false),
    LA_(32, true),  LA_(64, true),  LA_(128, true),  LA_(256, true),
};
static const Entry kLongB[] = {LB_(256, false), LB_(256, true)};
#undef LA_
#undef LB_

const Entry* findLongA(uint32_t n1, bool inverse) {
    for (const Entry& x : kLongA)
        if (x.n == n1 && x.flag == (int)inverse) return &x;
    return nullptr;
}
const Entry* findLongB(uint32_t n2, bool inverse) {
    for (const Entry& x : kLongB)
        if (x.n == n2 && x.flag == (int)inverse) return &x;
    return nullptr;
}

struct TwEntry {
    uint32_t n;
    int e;
    KTw fn;
    int count;
};
#define TW_(N, E) {N, E, &k_tw_stockham<N, E>, Sched<N, E>::TWSIZE}
static const TwEntry kTw[] = {
    TW_(16, 8), TW_(16, 16),
    TW_(32, 8), TW_(32, 16), TW_(64, 8), TW_(64, 16), TW_(128, 8), TW_(128, 16),
    TW_(256, 8), TW_(256, 16), TW_(512, 8), TW_(512, 16), TW_(1024, 8), TW_(1024, 16),
    TW_(2048, 8), TW_(2048, 16), TW_(4096, 8), TW_(4096, 16), TW_(8192, 8), TW_(8192, 16),
    TW_(16384, 8), TW_(16384, 16),
};
#undef TW_

bool findTw(uint32_t n, int e, KTw* fn, int* count) {
    for (const TwEntry& x : kTw)
        if (x.n == n && x.e == e) {
            *fn = x.fn;
            *count = x.count;
            return true;
        }
    return false;
}

}  // namespace dev
}  // namespace bfly
