// ref_wrap.cu -- C entry points that launch the reference's own multi-RHS hop kernels,
// compiled from their sources in the reference tree by oracle/ref_build.sh (test
// infrastructure; the product never loads the result).  Used once, on a GPU, to make
// the golden fixtures that pin the CPU oracle (tests/golden/make_golden.py).
//
//   ref_wmma_hop_f64  -> qcu::device::wilson_dslash_su_n_mrhs<double>
//                        (include/kernel/su_n_m_rhs_dslash.cuh:127-163; the kernel the
//                        reference's solver uses), launched as src/qcd/qcu_dslash_wilson.cu:20-33
//   ref_simt_hop_f64  -> qcu::device::wilson_dslash_su_n_mrhs<double, GemmShape<8,8,8>>
//                        (include/kernel/sun_mrhs_wilson_dslash_simt.cuh:203-228; the kernel of
//                        start_dslash / mat_Qcu), launched as src/qcd/qcu_wilson_dslash_simt.cu:33-66
#include <cuda_runtime.h>

#include "kernel/su_n_m_rhs_dslash.cuh"
#include "kernel/sun_mrhs_wilson_dslash_simt.cuh"

extern "C" int ref_wmma_hop_f64(double* out, const double* in, const double* gauge, const int* L, int n_color,
                                int m_rhs, int parity, int dagger) {
    const int half_vol = L[0] * L[1] * L[2] * L[3] / 2;
    dim3 block(WARP_SIZE, WARP_PER_BLOCK);
    dim3 grid(half_vol);
    qcu::device::wilson_dslash_su_n_mrhs<double><<<grid, block>>>(
        out, const_cast<double*>(in), const_cast<double*>(gauge), L[0], L[1], L[2], L[3], 1, 1, 1, 1, parity,
        dagger != 0, n_color, m_rhs);
    return (int)cudaDeviceSynchronize();
}

extern "C" int ref_simt_hop_f64(double* out, const double* in, const double* gauge, const int* L, int n_color,
                                int m_rhs, int parity, int dagger) {
    using BlockShape = qcu::gemm::GemmShape<8, 8, 8>;
    const int half_vol = L[0] * L[1] * L[2] * L[3] / 2;
    qcu::QcuLattDesc latt(L[0], L[1], L[2], L[3]);
    const int multiprocess = 0xF;   // process grid {1,1,1,1}: every dimension bit set
    dim3 grid(div_ceil(n_color, BlockShape::kM), div_ceil(m_rhs, BlockShape::kN), half_vol < 65535 ? half_vol : 65535);
    dim3 block(BlockShape::kM, BlockShape::kN, 1);
    qcu::device::wilson_dslash_su_n_mrhs<double, BlockShape><<<grid, block>>>(
        out, const_cast<double*>(in), const_cast<double*>(gauge), latt, multiprocess, parity, dagger != 0, n_color,
        m_rhs);
    return (int)cudaDeviceSynchronize();
}
