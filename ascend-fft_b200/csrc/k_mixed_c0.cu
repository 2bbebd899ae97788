// Instances of the mixed-radix kernels on the runtime pass list of radix class 0 (mixed.cuh).
#include "mixed.cuh"

namespace bfly {
namespace backend {
MixedKernels mixedGeneric0() { return kernelsOf<dev::GenericRows<0>>(); }
}  // namespace backend
}  // namespace bfly
