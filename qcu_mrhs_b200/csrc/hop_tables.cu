// hop_tables.cu -- per-site tables that the solver's tensor-core hop reads instead of
// recomputing them at every site of every hop:
//   * the neighbour table [2][Vh][8] (uint32): for output parity p and half-site x, the
//     half-site index of the forward and backward neighbour in x, y, z, t (the neighbour
//     rule of reference include/point/qcu_point.cuh:16-61, periodic in every direction);
//   * the hop-link array [2][Vh][4][2][N][N] complex in the storage precision: for output
//     parity p, site x and direction mu, W_f = U_mu(x) and W_b = U_mu(x - mu)^dag, both
//     multiplied by the t-boundary sign where the hop crosses the t boundary.  These are the
//     8 N x N link matrices each output site reads once (the links of the reference hop,
//     include/kernel/su_n_m_rhs_dslash.cuh:92-105, with the adjoint taken once per gauge
//     field instead of once per hop).
#include <algorithm>

#include "dslash.h"

namespace qcub {

namespace {

__global__ void neighbour_table_kernel(uint32_t* __restrict__ nbr, const Geom g) {
    const uint32_t vh = (uint32_t)g.vh;
    const uint32_t lxh = (uint32_t)g.lxh, Ly = (uint32_t)g.L[1], Lz = (uint32_t)g.L[2], Lt = (uint32_t)g.L[3];
    const uint32_t sy = lxh, sz = lxh * Ly, st = sz * Lz;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * vh; i += gridDim.x * blockDim.x) {
        const int parity = i >= vh;
        const uint32_t site = i - (parity ? vh : 0u);
        const SiteXYZT c = site_coords(g, site);
        const uint32_t xh = (uint32_t)c.xh;
        const int xodd = (parity ^ (c.y + c.z + c.t)) & 1;
        const uint32_t row = site - xh;
        uint4 a, b;
        a.x = row + (xodd ? (xh + 1 == lxh ? 0u : xh + 1) : xh);
        a.y = row + (xodd ? xh : (xh == 0 ? lxh - 1 : xh - 1));
        a.z = site + sy - ((uint32_t)c.y + 1 == Ly ? Ly * sy : 0u);
        a.w = site - sy + ((uint32_t)c.y == 0 ? Ly * sy : 0u);
        b.x = site + sz - ((uint32_t)c.z + 1 == Lz ? Lz * sz : 0u);
        b.y = site - sz + ((uint32_t)c.z == 0 ? Lz * sz : 0u);
        b.z = site + st - ((uint32_t)c.t + 1 == Lt ? Lt * st : 0u);
        b.w = site - st + ((uint32_t)c.t == 0 ? Lt * st : 0u);
        uint4* o = reinterpret_cast<uint4*>(nbr) + (size_t)i * 2;
        o[0] = a;
        o[1] = b;
    }
}

// One thread per (parity, site, mu, forward/backward, row c'): writes row c' of W.
template <typename S>
__global__ void hop_links_kernel(typename St<S>::S2* __restrict__ links, const typename St<S>::S2* __restrict__ gauge,
                                 const uint32_t* __restrict__ nbr, const Geom g, int nc, double t_sign) {
    using S2 = typename St<S>::S2;
    using A2 = typename St<S>::A2;
    using A = typename St<S>::A;
    const size_t vh = (size_t)g.vh;
    const size_t n2 = (size_t)nc * nc;
    const size_t total = 2 * vh * 8 * nc;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int cr = (int)(i % nc);
        const size_t e = i / nc;                 // (parity, site, hop)
        const int h = (int)(e % 8);
        const size_t ps = e / 8;                 // parity * vh + site
        const int parity = ps >= vh;
        const size_t site = ps - (parity ? vh : 0);
        const int mu = h >> 1;
        const bool fwd = (h & 1) == 0;
        const SiteXYZT c = site_coords(g, (uint32_t)site);
        const bool wrap = mu == 3 && (fwd ? (c.t + 1 == g.L[3]) : (c.t == 0));
        const A sg = wrap ? (A)t_sign : (A)1;
        S2* out = links + e * n2 + (size_t)cr * nc;
        if (fwd) {
            const S2* u = gauge + ((size_t)(mu * 2 + parity) * vh + site) * n2 + (size_t)cr * nc;
            for (int k = 0; k < nc; ++k) {
                const A2 v = St<S>::ld(u[k]);
                out[k] = St<S>::cv(mk2<A2>(sg * v.x, sg * v.y));
            }
        } else {
            const size_t nb = nbr[ps * 8 + h];
            const S2* u = gauge + ((size_t)(mu * 2 + (1 - parity)) * vh + nb) * n2 + cr;
            for (int k = 0; k < nc; ++k) {   // W_b[cr][k] = conj(U[k][cr])
                const A2 v = St<S>::ld(u[(size_t)k * nc]);
                out[k] = St<S>::cv(mk2<A2>(sg * v.x, -sg * v.y));
            }
        }
    }
}

}  // namespace

size_t neighbour_table_bytes(const Geom& g) { return (size_t)g.vh * 2 * 8 * sizeof(uint32_t); }

size_t hop_links_bytes(const Geom& g, int nc, int prec) {
    return (size_t)g.vh * 2 * 8 * nc * nc * 2 * prec_bytes(prec);
}

int build_neighbour_table(uint32_t* nbr, size_t bytes, const Geom& g, cudaStream_t st) {
    if (g.vh >= ((int64_t)1 << 30)) return set_error(QCU_ERR_UNSUPPORTED, "neighbour table: half volume beyond 2^30");
    if (!nbr || bytes < neighbour_table_bytes(g))
        return set_error(QCU_ERR_INVALID, "neighbour table: %zu bytes given, %zu needed", bytes,
                         neighbour_table_bytes(g));
    const int64_t n = 2 * g.vh;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 8 * sm_count());
    neighbour_table_kernel<<<grid, 256, 0, st>>>(nbr, g);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int build_hop_links(void* links, size_t bytes, const void* gauge, const uint32_t* nbr, const Geom& g, int nc,
                    int prec, double t_sign, cudaStream_t st) {
    if (!prec_valid(prec)) return set_error(QCU_ERR_INVALID, "hop links: precision %d", prec);
    if (!links || !gauge || !nbr || bytes < hop_links_bytes(g, nc, prec))
        return set_error(QCU_ERR_INVALID, "hop links: %zu bytes given, %zu needed", bytes, hop_links_bytes(g, nc, prec));
    const int64_t n = 2 * g.vh * 8 * nc;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 8 * sm_count());
    return dispatch_prec(prec, [&](auto tag) -> int {
        using S = decltype(tag);
        using S2 = typename St<S>::S2;
        hop_links_kernel<S><<<grid, 256, 0, st>>>(static_cast<S2*>(links), static_cast<const S2*>(gauge), nbr, g, nc,
                                                  t_sign);
        QCUB_CHECK_LAUNCH();
        return QCU_SUCCESS;
    });
}

}  // namespace qcub
