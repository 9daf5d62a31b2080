// dslash.h -- internal host API of the hop kernels.
#pragma once

#include "common.cuh"
#include "dslash_impl.cuh"

namespace qcub {

// Launch the hop kernel for colour count nc and storage precision prec.
int hop_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st);

}  // namespace qcub
