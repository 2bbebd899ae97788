// Instances of the mixed-radix kernels for plans fixed at compile time (mixed.cuh): common
// lengths (multiples of 10 and the half lengths of the real transforms of n = 320, 400, 480,
// 1000, 2000, 6000 ...; 7-smooth audio frame lengths 441, 882, 1764, 2205 and 7^4).
#include "mixed.cuh"

namespace bfly {
namespace backend {
namespace {
const FixedEntry kFixed[] = {
    BFLY_FIXED(15, 4),           // 60
    BFLY_FIXED(10, 10),          // 100
    BFLY_FIXED(15, 8),           // 120
    BFLY_FIXED(15, 10),          // 150
    BFLY_FIXED(16, 10),          // 160
    BFLY_FIXED(15, 12),          // 180
    BFLY_FIXED(10, 10, 2),       // 200
    BFLY_FIXED(16, 15),          // 240
    BFLY_FIXED(10, 5, 5),        // 250
    BFLY_FIXED(15, 10, 2),       // 300
    BFLY_FIXED(15, 12, 2),       // 360
    BFLY_FIXED(16, 5, 5),        // 400
    BFLY_FIXED(9, 7, 7),         // 441
    BFLY_FIXED(10, 10, 5),       // 500
    BFLY_FIXED(15, 9, 4),        // 540
    BFLY_FIXED(15, 10, 4),       // 600
    BFLY_FIXED(16, 15, 3),       // 720
    BFLY_FIXED(15, 10, 5),       // 750
    BFLY_FIXED(16, 10, 5),       // 800
    BFLY_FIXED(9, 14, 7),        // 882
    BFLY_FIXED(15, 15, 4),       // 900
    BFLY_FIXED(10, 10, 10),      // 1000
    BFLY_FIXED(16, 15, 5),       // 1200
    BFLY_FIXED(15, 10, 10),      // 1500
    BFLY_FIXED(9, 14, 14),       // 1764
    BFLY_FIXED(15, 15, 8),       // 1800
    BFLY_FIXED(16, 5, 5, 5),     // 2000
    BFLY_FIXED(15, 7, 7, 3),     // 2205
    BFLY_FIXED(16, 15, 10),      // 2400
    BFLY_FIXED(7, 7, 7, 7),      // 2401
    BFLY_FIXED(10, 10, 5, 5),    // 2500
    BFLY_FIXED(15, 10, 10, 2),   // 3000
    BFLY_FIXED(16, 15, 15),      // 3600
    BFLY_FIXED(16, 10, 5, 5),    // 4000
    BFLY_FIXED(10, 10, 10, 5),   // 5000
    BFLY_FIXED(16, 15, 5, 5),    // 6000
    BFLY_FIXED(9, 9, 9, 9),      // 6561
    BFLY_FIXED(16, 10, 10, 5),   // 8000
    BFLY_FIXED(10, 10, 10, 10),  // 10000
    BFLY_FIXED(16, 15, 10, 5),   // 12000
};
#undef BFLY_FIXED
}  // namespace

const FixedEntry* mixedFixed(int* count) {
    *count = (int)(sizeof(kFixed) / sizeof(kFixed[0]));
    return kFixed;
}
}  // namespace backend
}  // namespace bfly
