// Instances of the mixed-radix kernels on the runtime pass list of radix class 2 (mixed.cuh).
#include "mixed.cuh"

namespace bfly {
namespace backend {
MixedKernels mixedGeneric2() { return kernelsOf<dev::GenericRows<2>>(); }
}  // namespace backend
}  // namespace bfly
