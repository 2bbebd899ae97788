// Instances of the mixed-radix kernels on the runtime pass list of radix class 1 (mixed.cuh).
#include "mixed.cuh"

namespace bfly {
namespace backend {
MixedKernels mixedGeneric1() { return kernelsOf<dev::GenericRows<1>>(); }
}  // namespace backend
}  // namespace bfly
