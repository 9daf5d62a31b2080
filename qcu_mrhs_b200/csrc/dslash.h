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
// one-time set-up of the staged tensor-core hop (shared-memory opt-in, device error flag);
// call outside graph capture
int hop_mmal_prepare();

// per-site tables of the tensor-core hop (hop_tables.cu): neighbour table [2][Vh][8] and
// hop-link array [2][Vh][4][2][nc][nc] (W_f, W_b with the t-boundary sign folded in)
// (the builders check the destination's size in bytes against these)
size_t neighbour_table_bytes(const Geom& g);
size_t hop_links_bytes(const Geom& g, int nc, int prec);
int build_neighbour_table(uint32_t* nbr, size_t bytes, const Geom& g, cudaStream_t st);
int build_hop_links(void* links, size_t bytes, const void* gauge, const uint32_t* nbr, const Geom& g, int nc,
                    int prec, double t_sign, cudaStream_t st);
// whether the hop that hop_launch picks for (nc, m, prec) reads those tables
bool hop_reads_tables(int nc, int m, int prec);

// the kernel kind forced by qcuSetHopKernel (QCU_HOP_AUTO: none), and the automatic choice
// (tuner record, else the static rule) for a shape
int hop_kind();
int auto_hop_kind(int nc, int m, int prec);

}  // namespace qcub
