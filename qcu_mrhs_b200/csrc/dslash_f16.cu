// dslash_f16.cu -- hop kernels with __half storage (instantiations only; see dslash_impl.cuh).
#include "dslash_launch.cuh"

namespace qcub {
QCUB_INSTANTIATE_HOP(__half)
}  // namespace qcub
