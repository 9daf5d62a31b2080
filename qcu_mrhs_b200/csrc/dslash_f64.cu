// dslash_f64.cu -- hop kernels with double storage (instantiations only; see dslash_impl.cuh).
#include "dslash_launch.cuh"

namespace qcub {
QCUB_INSTANTIATE_HOP(double)
}  // namespace qcub
