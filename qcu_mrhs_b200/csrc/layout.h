// layout.h -- internal host API of the layout kernels.
#pragma once

#include "common.cuh"

namespace qcub {

// src/dst: HOST arrays of m device pointers to per-RHS single-parity fields [Vh][4][nc]
int gather_mrhs(void* dst, int dprec, void* const* src, int sprec, int64_t vh, int nc, int m,
                cudaStream_t st);
int scatter_mrhs(void* const* dst, int dprec, const void* src, int sprec, int64_t vh, int nc, int m,
                 cudaStream_t st);
int cast_complex(void* dst, int dprec, const void* src, int sprec, int64_t n, cudaStream_t st);
// to_eo = 1: lexicographic -> even/odd; 0: even/odd -> lexicographic
int gauge_reorder(void* dst, const void* src, const int L[4], int nc, int prec, int to_eo,
                  cudaStream_t st);
// fermion [Lt][Lz][Ly][Lx][4][nc] <-> [2][Vh][4][nc]
int fermion_reorder(void* dst, const void* src, const int L[4], int nc, int prec, int to_eo, cudaStream_t st);
// multi-RHS half-lattice field: gathered [Vh][4nc][m] <-> site-blocked (kSiteBlock)
int site_block_reorder(void* dst, const void* src, int64_t vh, int nc, int m, int prec, int to_blocked,
                       cudaStream_t st);

}  // namespace qcub
