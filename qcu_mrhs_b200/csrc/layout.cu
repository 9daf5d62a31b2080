// layout.cu -- per-RHS <-> gathered multi-RHS transposition, precision casts,
// lexicographic <-> even/odd gauge reorder.
//
// Gather/scatter replace reference include/kernel/copy_vector/copy_color_spinor.cuh:16-102
// (one thread per site looping over m x Ns x Nc with stride-m stores, plus an H2D copy
// of the pointer table per call, src/qcu_interface.cu:123-126).  Here a block stages a
// tile of sites of all m RHS in shared memory: it reads each RHS's contiguous run and
// writes the RHS-fastest output contiguously.  The m pointers travel as a kernel argument.
#include "layout.h"

namespace qcub {

struct PtrTable {
    void* p[kMaxRhs];
};

constexpr int kTileBytes = 32768;
constexpr int kLayoutThreads = 256;

// tile sites so that m * ts * site_len complex values of the arithmetic type fit
template <typename A2>
static int tile_sites(int m, int site_len) {
    int ts = kTileBytes / (int)(sizeof(A2) * m * site_len);
    return ts < 1 ? 1 : ts;
}

template <typename D, typename S>
__global__ void __launch_bounds__(kLayoutThreads)
gather_kernel(typename St<D>::S2* __restrict__ dst, PtrTable src, int64_t vh, int site_len, int m,
              int ts) {
    using A2 = typename St<S>::A2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A2* tile = reinterpret_cast<A2*>(smem_raw);
    const int run = ts * site_len;      // complex values per RHS in the tile
    const int ld = run + 1;             // padded row
    for (int64_t s0 = (int64_t)blockIdx.x * ts; s0 < vh; s0 += (int64_t)gridDim.x * ts) {
        const int nsite = (int)((vh - s0) < ts ? (vh - s0) : ts);
        const int nrun = nsite * site_len;
        for (int idx = threadIdx.x; idx < m * nrun; idx += blockDim.x) {
            const int r = idx / nrun, k = idx - r * nrun;
            const typename St<S>::S2* sp = static_cast<const typename St<S>::S2*>(src.p[r]);
            tile[r * ld + k] = St<S>::ld(sp[s0 * site_len + k]);
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < m * nrun; idx += blockDim.x) {
            const int k = idx / m, r = idx - k * m;
            const A2 v = tile[r * ld + k];
            typename St<D>::A2 d;
            d.x = (typename St<D>::A)v.x;
            d.y = (typename St<D>::A)v.y;
            dst[(s0 * site_len) * m + idx] = St<D>::cv(d);
        }
        __syncthreads();
    }
}

template <typename D, typename S>
__global__ void __launch_bounds__(kLayoutThreads)
scatter_kernel(PtrTable dst, const typename St<S>::S2* __restrict__ src, int64_t vh, int site_len,
               int m, int ts) {
    using A2 = typename St<S>::A2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A2* tile = reinterpret_cast<A2*>(smem_raw);
    const int run = ts * site_len;
    const int ld = run + 1;
    for (int64_t s0 = (int64_t)blockIdx.x * ts; s0 < vh; s0 += (int64_t)gridDim.x * ts) {
        const int nsite = (int)((vh - s0) < ts ? (vh - s0) : ts);
        const int nrun = nsite * site_len;
        for (int idx = threadIdx.x; idx < m * nrun; idx += blockDim.x) {
            const int k = idx / m, r = idx - k * m;
            tile[r * ld + k] = St<S>::ld(src[(s0 * site_len) * m + idx]);
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < m * nrun; idx += blockDim.x) {
            const int r = idx / nrun, k = idx - r * nrun;
            const A2 v = tile[r * ld + k];
            typename St<D>::A2 d;
            d.x = (typename St<D>::A)v.x;
            d.y = (typename St<D>::A)v.y;
            static_cast<typename St<D>::S2*>(dst.p[r])[s0 * site_len + k] = St<D>::cv(d);
        }
        __syncthreads();
    }
}

template <typename D, typename S>
__global__ void cast_kernel(typename St<D>::S2* __restrict__ dst, const typename St<S>::S2* __restrict__ src,
                            int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = convert2<D, S>(src[i]);
}

// lexicographic [4][Lt][Lz][Ly][Lx][N][N] <-> even/odd [4][2][Vh][N][N]
// Site reorder between lexicographic [nblk][Lt][Lz][Ly][Lx][per_site] and even/odd
// [nblk][2][Vh][per_site] (parity (x+y+z+t) mod 2, full x = 2 xh + ((p + y + z + t) & 1)):
// the gauge field has 4 blocks (directions) of N*N per site, a fermion 1 block of 4*N.
template <typename S>
__global__ void site_reorder_kernel(typename St<S>::S2* __restrict__ dst, const typename St<S>::S2* __restrict__ src,
                                    Geom g, int per_site, int nblk, int to_eo) {
    const int64_t V = 2 * g.vh;
    const int64_t total = (int64_t)nblk * V * per_site;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        // i indexes the even/odd array
        const int e = (int)(i % per_site);
        int64_t q = i / per_site;
        const int64_t hidx = q % g.vh;
        q /= g.vh;
        const int par = (int)(q % 2);
        const int blk = (int)(q / 2);
        int64_t h = hidx;
        const int xh = (int)(h % g.lxh); h /= g.lxh;
        const int y = (int)(h % g.L[1]); h /= g.L[1];
        const int z = (int)(h % g.L[2]);
        const int t = (int)(h / g.L[2]);
        const int x = 2 * xh + ((par + y + z + t) & 1);
        const int64_t lex = (((int64_t)t * g.L[2] + z) * g.L[1] + y) * g.L[0] + x;
        const int64_t li = ((int64_t)blk * V + lex) * per_site + e;
        if (to_eo) dst[i] = src[li];
        else dst[li] = src[i];
    }
}

template <typename D, typename S>
static int gather_t(void* dst, void* const* src, int64_t vh, int nc, int m, cudaStream_t st) {
    PtrTable t{};
    for (int r = 0; r < m; ++r) t.p[r] = src[r];
    const int sl = kNs * nc;
    using A2 = typename St<S>::A2;
    const int ts = tile_sites<A2>(m, sl);
    const size_t smem = sizeof(A2) * (size_t)m * (ts * sl + 1);
    auto k = gather_kernel<D, S>;
    if (smem > 48 * 1024) QCUB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t tiles = (vh + ts - 1) / ts;
    const int grid = (int)(tiles < 65535 * 4 ? tiles : 65535 * 4);
    k<<<grid, kLayoutThreads, smem, st>>>(static_cast<typename St<D>::S2*>(dst), t, vh, sl, m, ts);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <typename D, typename S>
static int scatter_t(void* const* dst, const void* src, int64_t vh, int nc, int m, cudaStream_t st) {
    PtrTable t{};
    for (int r = 0; r < m; ++r) t.p[r] = dst[r];
    const int sl = kNs * nc;
    using A2 = typename St<S>::A2;
    const int ts = tile_sites<A2>(m, sl);
    const size_t smem = sizeof(A2) * (size_t)m * (ts * sl + 1);
    auto k = scatter_kernel<D, S>;
    if (smem > 48 * 1024) QCUB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t tiles = (vh + ts - 1) / ts;
    const int grid = (int)(tiles < 65535 * 4 ? tiles : 65535 * 4);
    k<<<grid, kLayoutThreads, smem, st>>>(t, static_cast<const typename St<S>::S2*>(src), vh, sl, m, ts);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int gather_mrhs(void* dst, int dprec, void* const* src, int sprec, int64_t vh, int nc, int m,
                cudaStream_t st) {
    if (m < 1 || m > kMaxRhs) return set_error(QCU_ERR_INVALID, "m_rhs=%d", m);
    if (nc < 1 || nc > kMaxColor) return set_error(QCU_ERR_INVALID, "n_color=%d", nc);
    for (int r = 0; r < m; ++r)
        if (src[r] == nullptr) return set_error(QCU_ERR_INVALID, "null fermion pointer %d", r);
    return dispatch_prec(dprec, [&](auto dt) {
        return dispatch_prec(sprec, [&](auto stt) {
            return gather_t<decltype(dt), decltype(stt)>(dst, src, vh, nc, m, st);
        });
    });
}

int scatter_mrhs(void* const* dst, int dprec, const void* src, int sprec, int64_t vh, int nc, int m,
                 cudaStream_t st) {
    if (m < 1 || m > kMaxRhs) return set_error(QCU_ERR_INVALID, "m_rhs=%d", m);
    if (nc < 1 || nc > kMaxColor) return set_error(QCU_ERR_INVALID, "n_color=%d", nc);
    for (int r = 0; r < m; ++r)
        if (dst[r] == nullptr) return set_error(QCU_ERR_INVALID, "null fermion pointer %d", r);
    return dispatch_prec(dprec, [&](auto dt) {
        return dispatch_prec(sprec, [&](auto stt) {
            return scatter_t<decltype(dt), decltype(stt)>(dst, src, vh, nc, m, st);
        });
    });
}

int cast_complex(void* dst, int dprec, const void* src, int sprec, int64_t n, cudaStream_t st) {
    if (n < 0) return set_error(QCU_ERR_INVALID, "negative length");
    if (n == 0) return QCU_SUCCESS;
    return dispatch_prec(dprec, [&](auto dt) {
        return dispatch_prec(sprec, [&](auto stt) {
            using D = decltype(dt);
            using S = decltype(stt);
            auto k = cast_kernel<D, S>;
            const int grid = resident_grid(k, 256, n);
            k<<<grid, 256, 0, st>>>(static_cast<typename St<D>::S2*>(dst),
                                    static_cast<const typename St<S>::S2*>(src), n);
            QCUB_CHECK_LAUNCH();
            return QCU_SUCCESS;
        });
    });
}

static int site_reorder(void* dst, const void* src, const int L[4], int per_site, int nblk, int prec, int to_eo,
                        cudaStream_t st) {
    if (L[0] < 2 || L[0] % 2 || L[1] < 1 || L[2] < 1 || L[3] < 1)
        return set_error(QCU_ERR_INVALID, "lattice %dx%dx%dx%d (Lx must be even)", L[0], L[1], L[2], L[3]);
    if (dst == src) return set_error(QCU_ERR_INVALID, "in-place reorder is not supported");
    const Geom g = make_geom(L);
    return dispatch_prec(prec, [&](auto tag) {
        using S = decltype(tag);
        auto k = site_reorder_kernel<S>;
        const int grid = resident_grid(k, 256, 2 * g.vh * nblk * per_site);
        k<<<grid, 256, 0, st>>>(static_cast<typename St<S>::S2*>(dst), static_cast<const typename St<S>::S2*>(src), g,
                                per_site, nblk, to_eo);
        QCUB_CHECK_LAUNCH();
        return QCU_SUCCESS;
    });
}

int gauge_reorder(void* dst, const void* src, const int L[4], int nc, int prec, int to_eo, cudaStream_t st) {
    return site_reorder(dst, src, L, nc * nc, 4, prec, to_eo, st);
}

// gathered [Vh][4N][m] <-> site-blocked (kSiteBlock) multi-RHS half-lattice field
template <typename S>
__global__ void site_block_kernel(typename St<S>::S2* __restrict__ dst, const typename St<S>::S2* __restrict__ src,
                                  int64_t n, int m, int rows, int to_blocked) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = site_blocked_index(i, m, rows);
        if (to_blocked) dst[b] = src[i];
        else dst[i] = src[b];
    }
}

int site_block_reorder(void* dst, const void* src, int64_t vh, int nc, int m, int prec, int to_blocked,
                       cudaStream_t st) {
    if (!dst || !src) return set_error(QCU_ERR_INVALID, "null pointer");
    if (dst == src) return set_error(QCU_ERR_INVALID, "the site-blocked reorder cannot run in place");
    if (nc < 1 || nc > kMaxColor || m < 1 || m > kMaxRhs)
        return set_error(QCU_ERR_INVALID, "n_color=%d m_rhs=%d", nc, m);
    if (vh < 1 || vh % kSiteBlock)
        return set_error(QCU_ERR_INVALID, "half volume %lld is not a multiple of %d", (long long)vh, kSiteBlock);
    const int64_t n = vh * 4 * nc * m;
    if (n >= ((int64_t)1 << 31)) return set_error(QCU_ERR_UNSUPPORTED, "site-blocked field beyond 2^31 complex");
    return dispatch_prec(prec, [&](auto tag) -> int {
        using S = decltype(tag);
        auto k = site_block_kernel<S>;
        const int grid = resident_grid(k, kLayoutThreads, n);
        k<<<grid, kLayoutThreads, 0, st>>>(static_cast<typename St<S>::S2*>(dst),
                                           static_cast<const typename St<S>::S2*>(src), n, m, 4 * nc, to_blocked);
        QCUB_CHECK_LAUNCH();
        return QCU_SUCCESS;
    });
}

int fermion_reorder(void* dst, const void* src, const int L[4], int nc, int prec, int to_eo, cudaStream_t st) {
    return site_reorder(dst, src, L, 4 * nc, 1, prec, to_eo, st);
}

}  // namespace qcub
