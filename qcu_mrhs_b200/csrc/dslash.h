// dslash.h -- internal host API of the hop kernels.
#pragma once

#include "common.cuh"
#include "dslash_impl.cuh"

namespace qcub {

// Launch the hop kernel for colour count nc and storage precision prec.
// p.blocked routes to the two-RHS packed 16-bit kernel, the one kernel that reads the
// site-blocked layout.
int hop_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st);

// two-RHS packed 16-bit kernel: SU(3), m = 8, 12, 16; the site-blocked layout further needs
// a half volume that is a multiple of kSiteBlock and fewer than 2^31 complex per vector
bool hop16_pairs_supported(int nc, int m, int prec);
bool hop16_blocked_supported(int nc, int m, int prec, int64_t vh);
// one-time kernel attributes of the two-RHS kernel; call outside graph capture
int hop16_pairs_prepare();

// the kernel kind forced by qcuSetHopKernel (QCU_HOP_AUTO: none), and the automatic choice
// (tuner record, else the static rule) for a shape
int hop_kind();
int auto_hop_kind(int nc, int m, int prec);

}  // namespace qcub
