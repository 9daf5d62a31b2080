// dslash_bf16.cu -- hop kernels with __nv_bfloat16 storage (instantiations only; see dslash_impl.cuh).
#include "dslash_launch.cuh"

namespace qcub {
QCUB_INSTANTIATE_HOP(__nv_bfloat16)
}  // namespace qcub
