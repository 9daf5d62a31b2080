// dslash_launch.cuh -- host launcher for hop_kernel instantiations.
#pragma once

#include "dslash_impl.cuh"
#include "workspace.h"

namespace qcub {

template <int NC, typename S>
int launch_hop(const HopParams& p, bool dagger, int epi, cudaStream_t stream, bool color_split) {
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    void (*k)(const HopParams) = nullptr;
    if (color_split) {
        switch (epi) {
            case EPI_PLAIN: k = dagger ? hop_kernel_cs<NC, S, true, EPI_PLAIN> : hop_kernel_cs<NC, S, false, EPI_PLAIN>; break;
            case EPI_XPAY: k = dagger ? hop_kernel_cs<NC, S, true, EPI_XPAY> : hop_kernel_cs<NC, S, false, EPI_XPAY>; break;
            case EPI_SCHUR_R0: k = hop_kernel_cs<NC, S, false, EPI_SCHUR_R0>; break;
            case EPI_SCHUR_TS: k = hop_kernel_cs<NC, S, false, EPI_SCHUR_TS>; break;
            case EPI_SCHUR: k = hop_kernel_cs<NC, S, false, EPI_SCHUR>; break;
            case EPI_RESID: k = hop_kernel_cs<NC, S, false, EPI_RESID>; break;
            default: return set_error(QCU_ERR_INVALID, "unknown hop epilogue %d", epi);
        }
    } else {
        switch (epi) {
            case EPI_PLAIN: k = dagger ? hop_kernel<NC, S, true, EPI_PLAIN> : hop_kernel<NC, S, false, EPI_PLAIN>; break;
            case EPI_XPAY: k = dagger ? hop_kernel<NC, S, true, EPI_XPAY> : hop_kernel<NC, S, false, EPI_XPAY>; break;
            case EPI_SCHUR_R0: k = hop_kernel<NC, S, false, EPI_SCHUR_R0>; break;
            case EPI_SCHUR_TS: k = hop_kernel<NC, S, false, EPI_SCHUR_TS>; break;
            case EPI_SCHUR: k = hop_kernel<NC, S, false, EPI_SCHUR>; break;
            case EPI_RESID: k = hop_kernel<NC, S, false, EPI_RESID>; break;
            default: return set_error(QCU_ERR_INVALID, "unknown hop epilogue %d", epi);
        }
    }
    // block: a multiple of the threads of one site (m, or N*m when the colour is split)
    const int per = color_split ? NC * p.m : p.m;
    const int block = (kRedThreads / per) * per;
    const int64_t total = p.g.vh * per;
    int grid = resident_grid(k, block, total);
    if (grid > kScratchBlocks) grid = kScratchBlocks;   // partial sums fit the scratch
    k<<<grid, block, 0, stream>>>(p);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

#define QCUB_INSTANTIATE_HOP(S)                                                          \
    template int launch_hop<2, S>(const HopParams&, bool, int, cudaStream_t, bool);            \
    template int launch_hop<3, S>(const HopParams&, bool, int, cudaStream_t, bool);            \
    template int launch_hop<4, S>(const HopParams&, bool, int, cudaStream_t, bool);            \
    template int launch_hop<5, S>(const HopParams&, bool, int, cudaStream_t, bool);            \
    template int launch_hop<6, S>(const HopParams&, bool, int, cudaStream_t, bool);            \
    template int launch_hop<7, S>(const HopParams&, bool, int, cudaStream_t, bool);            \
    template int launch_hop<8, S>(const HopParams&, bool, int, cudaStream_t, bool);

}  // namespace qcub
