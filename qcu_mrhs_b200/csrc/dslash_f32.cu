// dslash_f32.cu -- hop kernels with float storage (instantiations only; see dslash_impl.cuh).
#include "dslash_launch.cuh"

namespace qcub {
QCUB_INSTANTIATE_HOP(float)
}  // namespace qcub
