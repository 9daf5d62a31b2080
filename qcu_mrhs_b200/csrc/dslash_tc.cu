// dslash_tc.cu -- multi-RHS hop term on the 5th-generation tensor cores (tcgen05),
// for FP16 and BF16 storage with FP32 accumulation in tensor memory.
//
// Same operator and layouts as dslash_impl.cuh (reference
// include/kernel/su_n_m_rhs_dslash.cuh:92-105, complex_matmul.cuh:16-600).
//
// The kernel (hop_mma_kernel, below) turns the 8 hops of a site into one real GEMM with
// K = 8 hops x 2N: A rows are the projected neighbour spinors (spin, RHS), B the real
// embedding of the 8 link matrices.  A and B are written to shared memory by the CTA's
// threads; tcgen05.mma kind::f16 (M = 128, N = 16, K = 16, issued by one thread) sums
// into tensor memory; completion is signalled through tcgen05.commit to an mbarrier.
// Every wait on an mbarrier is bounded; on timeout the kernel records an error code and
// finishes (results are then invalid, never a hang).
#include "dslash.h"
#include "dslash_impl.cuh"
#include "workspace.h"

namespace qcub {

int* device_error_flag();   // runtime.cu: per-device flag, nonzero after a timed-out wait

namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for the phase with the given parity to complete: gives up after ~2^30 SM
// cycles (about half a second) and returns false.  Callers stop waiting once a wait has
// failed, so a kernel whose pipeline broke finishes quickly with its error flag set.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > (1ll << 30)) return false;
    }
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// K-major, no-swizzle shared-memory matrix descriptor: 8-row x 16-byte core matrices,
// LBO = byte distance between the two K-adjacent core matrices, SBO = between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(const void* base, uint32_t lbo, uint32_t sbo) {
    const uint64_t addr = smem_u32(base);
    return ((addr >> 4) & 0x3FFFull) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16, D = F32, A/B = F16 (fmt 0) or BF16 (fmt 1), both
// K-major, M = 128, N = 16.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

template <typename S> struct Pk;
template <> struct Pk<__half> {
    using T2 = __half2;
    static constexpr uint32_t fmt = 0;
    __device__ static T2 sgn(float a, float b) { return __floats2half2_rn(a, b); }
};
template <> struct Pk<__nv_bfloat16> {
    using T2 = __nv_bfloat162;
    static constexpr uint32_t fmt = 1;
    __device__ static T2 sgn(float a, float b) { return __floats2bfloat162_rn(a, b); }
};

template <typename T2>
__device__ __forceinline__ uint32_t as_u32(T2 v) {
    return *reinterpret_cast<uint32_t*>(&v);
}
template <typename T2>
__device__ __forceinline__ T2 from_u32(uint32_t u) {
    return *reinterpret_cast<T2*>(&u);
}

struct Tile {
    int lxh, Ly, Lz, Lt;
    int64_t vh;
};

// neighbour half-site index of `site` (parity `parity`) in direction mu, forward/backward;
// *wrap is set when the hop crosses the t boundary.
__device__ __forceinline__ int64_t neighbour(const Tile& g, int64_t site, int xh, int y, int z, int t,
                                             int xodd, int mu, bool fwd, bool* wrap) {
    const int64_t sy = g.lxh, sz = (int64_t)g.lxh * g.Ly, st = sz * g.Lz;
    *wrap = false;
    switch (mu) {
        case 0:
            if (fwd) return site - xh + (xodd ? (xh + 1 == g.lxh ? 0 : xh + 1) : xh);
            return site - xh + (xodd ? xh : (xh == 0 ? g.lxh - 1 : xh - 1));
        case 1:
            if (fwd) return site + (y + 1 == g.Ly ? -(int64_t)(g.Ly - 1) * sy : sy);
            return site + (y == 0 ? (int64_t)(g.Ly - 1) * sy : -sy);
        case 2:
            if (fwd) return site + (z + 1 == g.Lz ? -(int64_t)(g.Lz - 1) * sz : sz);
            return site + (z == 0 ? (int64_t)(g.Lz - 1) * sz : -sz);
        default:
            if (fwd) {
                *wrap = (t + 1 == g.Lt);
                return site + (*wrap ? -(int64_t)(g.Lt - 1) * st : st);
            }
            *wrap = (t == 0);
            return site + (*wrap ? (int64_t)(g.Lt - 1) * st : -st);
    }
}

struct SiteCoord {
    int xh, y, z, t, xodd;
};

__device__ __forceinline__ SiteCoord coords(const Geom& geo, int64_t site, int parity) {
    const SiteXYZT q = site_coords(geo, (uint32_t)site);
    SiteCoord c;
    c.xh = q.xh;
    c.y = q.y;
    c.z = q.z;
    c.t = q.t;
    c.xodd = (parity ^ (c.y + c.z + c.t)) & 1;
    return c;
}

// =====================================================================================
// One GEMM per pair of sites (hop_mma_kernel) -- the kernel behind QCU_HOP_TENSOR.
//
// For a site x the 8 hops form one real matrix product:
//   out[s'][c][r] = sum_{h, c', ri} A[(s', r)][(h, c', ri)] * B[(h, c', ri)][(c, ro)]
//   A row (s', r): the projected neighbour spinor of every hop,
//       R_h[s'][c'][r] = psi_{x+h}[s'][c'][r] + coef_h(s') psi_{x+h}[p_h(s')][c'][r];
//   B: the real embedding of W_h^T (W_h = U_mu(x) forward, U_mu(x - mu)^dag backward;
//       column (c, re) holds (Re W, -Im W) over (c', re/im), column (c, im) (Im W, Re W)).
// K = 8 hops x 2N = 16N: N MMAs of K = 16 per tile.  Two sites share an M = 128 tile
// (rows 0..4m-1 site a, 4m..8m-1 site b) and B = [B_a | B_b] (8 columns each), so site a's
// rows read columns 0..7 of D and site b's rows columns 8..15 (no block-diagonal zeros).
// A and B live in shared memory (K-major, no swizzle); D (128 lanes x 16 FP32 columns per
// tile) in tensor memory.  A CTA of 128 threads processes T tiles per round: the threads
// write A and B, one thread issues the T x N MMAs and a commit, every thread waits on the
// commit's mbarrier (bounded), then reads its own TMEM lane (= its A row) and writes it.
// =====================================================================================
constexpr int kMmaThreads = 128;
constexpr int kMmaMaxTiles = 5;
constexpr int kMmaTmemCols = 128;   // T x 16 <= 80 columns used

// Partner spin p(s) and sign of gamma_mu[s][p(s)] in the DeGrand-Rossi basis (reference
// include/kernel/qcu_gamma.cuh): mu=0: +i,+i,-i,-i ; mu=1: -1,+1,+1,-1 ; mu=2: +i,-i,-i,+i ;
// mu=3: +1,+1,+1,+1 (gamma_1 and gamma_3 entries are imaginary); nibble mu of 0x069C has
// bit s set where the entry is negative.
__host__ __device__ constexpr int gsign_c(int mu, int s) { return ((0x069C >> (4 * mu + s)) & 1) ? -1 : 1; }
__host__ __device__ constexpr int partner_c(int mu, int s) { return mu < 2 ? 3 - s : (s ^ 2); }

struct MmaPlan {
    int S;          // sites per tile (2 when 8m <= 128)
    int T;          // tiles per round
    int K;          // 16 N
    int a_bytes;    // 128 x K 16-bit values
    int b_bytes;    // 16 x K 16-bit values
};
__host__ __device__ inline MmaPlan mma_plan(int nc, int m) {
    MmaPlan q;
    q.S = (8 * m <= 128) ? 2 : 1;
    q.K = 16 * nc;
    const int per_tile = q.S * m;
    q.T = kMmaThreads / per_tile;
    if (q.T > kMmaMaxTiles) q.T = kMmaMaxTiles;
    if (q.T < 1) q.T = 1;
    q.a_bytes = 128 * q.K * 2;
    q.b_bytes = 16 * q.K * 2;
    return q;
}
inline size_t mma_smem_bytes(int nc, int m) {
    const MmaPlan q = mma_plan(nc, m);
    return (size_t)q.T * (q.a_bytes + q.b_bytes);
}

// byte offset of (row n, k) in a K-major, no-swizzle operand with R row groups:
// core matrix (n / 8, k / 8) at ((k / 8) * R + n / 8) * 128, row n % 8 at +16, k % 8 at +2
__device__ __forceinline__ uint32_t kmajor_off(int n, int k, int row_groups) {
    return (uint32_t)((((k >> 3) * row_groups + (n >> 3)) << 7) + ((n & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ void mma_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// packed-word helpers (re low half, im high half)
__device__ __forceinline__ uint32_t w_times_i(uint32_t u) { return __byte_perm(u, 0, 0x1032) ^ 0x00008000u; }
__device__ __forceinline__ uint32_t w_times_mi(uint32_t u) { return __byte_perm(u, 0, 0x1032) ^ 0x80000000u; }

template <typename S>
__device__ __forceinline__ uint32_t w_add(uint32_t a, uint32_t b) {
    return as_u32(__hadd2(from_u32<typename Pk<S>::T2>(a), from_u32<typename Pk<S>::T2>(b)));
}

// a + cs * (imag ? i b : b), cs = +-1 known at compile time
template <typename S, int CS, bool IMAG>
__device__ __forceinline__ uint32_t w_project(uint32_t a, uint32_t b) {
    uint32_t t;
    if (IMAG) t = CS > 0 ? w_times_i(b) : w_times_mi(b);
    else t = CS > 0 ? b : (b ^ 0x80008000u);
    return w_add<S>(a, t);
}

template <int NC, typename S, bool DAG, int H>
__device__ __forceinline__ void mma_rows_hop(uint32_t (&rw)[4][4 * NC], const uint32_t* __restrict__ src, int m) {
    constexpr int MU = H >> 1;
    constexpr bool FWD = (H & 1) == 0;
    constexpr bool IMAG = (MU == 0 || MU == 2);
    constexpr int SG = FWD ? (DAG ? 1 : -1) : (DAG ? -1 : 1);   // 1 + SG gamma_mu
    uint32_t v[4][NC];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < NC; ++c) v[s][c] = __ldg(src + (s * NC + c) * m);
    constexpr int hl = H & 3;   // position of the hop in its group of 4
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        rw[0][hl * NC + c] = w_project<S, SG * gsign_c(MU, 0), IMAG>(v[0][c], v[partner_c(MU, 0)][c]);
        rw[1][hl * NC + c] = w_project<S, SG * gsign_c(MU, 1), IMAG>(v[1][c], v[partner_c(MU, 1)][c]);
        rw[2][hl * NC + c] = w_project<S, SG * gsign_c(MU, 2), IMAG>(v[2][c], v[partner_c(MU, 2)][c]);
        rw[3][hl * NC + c] = w_project<S, SG * gsign_c(MU, 3), IMAG>(v[3][c], v[partner_c(MU, 3)][c]);
    }
}

template <int NC, typename S, bool DAG, int EPI>
__global__ void __launch_bounds__(kMmaThreads) hop_mma_kernel(const HopParams p, int* err) {
    using S2 = typename St<S>::S2;
    using A2 = typename St<S>::A2;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int N2 = NC * NC;
    extern __shared__ __align__(128) uint8_t smem8[];
    __shared__ __align__(8) uint64_t sMma;
    __shared__ uint32_t sTmem;
    __shared__ int sNb[kMmaMaxTiles][2][8];
    __shared__ int sAbort;

    if (skip_launch(p.done, p.gate)) return;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int m = p.m;
    const MmaPlan plan = mma_plan(NC, m);
    const int S_ = plan.S, T = plan.T;
    const int rows_used = S_ * 4 * m;
    const int64_t vh = p.g.vh;
    const int parity = p.parity;
    const int64_t site_len = (int64_t)kNs * NC * m;
    const int64_t per_round = (int64_t)T * S_;
    const int64_t nrounds = (vh + per_round - 1) / per_round;
    const uint32_t* __restrict__ in = static_cast<const uint32_t*>(p.in);
    const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
    const int64_t gmu = 2 * vh * N2;
    const uint32_t tflip = p.t_sign < 0 ? 0x80008000u : 0u;
    uint8_t* sA = smem8;                                   // T tiles of a_bytes
    uint8_t* sB = smem8 + (size_t)T * plan.a_bytes;        // T tiles of b_bytes

    // ---- set-up: zero A and B once (unused rows / columns stay zero), TMEM, mbarrier ----
    {
        uint4* z = reinterpret_cast<uint4*>(smem8);
        const int n16 = T * (plan.a_bytes + plan.b_bytes) / 16;
        for (int i = tid; i < n16; i += kMmaThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (tid == 0) {
        mbar_init(&sMma, 1);
        sAbort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sTmem)),
                     "r"(kMmaTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = sTmem;
    const uint32_t idesc = instr_desc(Pk<S>::fmt);   // M = 128, N = 16, K-major A and B

    // producer role of this thread: (tile, slot, RHS)
    const int per_tile = S_ * m;
    const int pt = tid / per_tile;
    const int pslot = (tid % per_tile) / m;
    const int prr = tid % m;
    const bool producer = pt < T;
    // epilogue role: TMEM lane = A row = tid
    const bool row_used = tid < rows_used;
    const int eslot = row_used ? tid / (4 * m) : 0;
    const int ewithin = tid - eslot * 4 * m;
    const int esp = row_used ? ewithin / m : 0;
    const int err_ = ewithin - esp * m;   // RHS of this row
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;

    A2 red[NV > 0 ? NV : 1];
#pragma unroll
    for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[k] = mk2<A2>(0, 0);
    uint32_t phase = 0;
    bool timed_out = false;

    for (int64_t round = blockIdx.x; round < nrounds; round += gridDim.x) {
        const int64_t base = round * per_round;
        // ---- neighbours of this thread's site (producers) ----
        int64_t psite = base + (int64_t)pt * S_ + pslot;
        const bool pvalid = producer && psite < vh;
        int64_t nbs[8];
        uint32_t wrapf = 0;
        if (pvalid) {
            const SiteCoord c = coords(p.g, psite, parity);
            const Tile tg{p.g.lxh, p.g.L[1], p.g.L[2], p.g.L[3], vh};
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                bool wrap;
                nbs[h] = neighbour(tg, psite, c.xh, c.y, c.z, c.t, c.xodd, h >> 1, (h & 1) == 0, &wrap);
                if (wrap) wrapf |= 1u << h;
            }
            if (prr == 0)
#pragma unroll
                for (int h = 0; h < 8; ++h) sNb[pt][pslot][h] = (int)nbs[h] | (((wrapf >> h) & 1u) ? (int)0x80000000u : 0);
        }
        __syncthreads();   // sNb visible; the previous round's epilogue has finished with TMEM
        // ---- B: real embedding of the links, T x S x 8 x N x N items of two words ----
        {
            const int nitems = T * S_ * 8 * N2;
            for (int it = tid; it < nitems; it += kMmaThreads) {
                int q = it;
                const int cc = q % NC; q /= NC;       // c'
                const int c = q % NC; q /= NC;        // c
                const int h = q % 8; q /= 8;
                const int sl = q % S_;
                const int t = q / S_;
                const int64_t site = base + (int64_t)t * S_ + sl;
                if (site >= vh) continue;
                const int mu = h >> 1;
                const int nbw = sNb[t][sl][h];
                uint32_t w;
                if ((h & 1) == 0) {
                    w = __ldg(gauge + (int64_t)parity * vh * N2 + mu * gmu + site * N2 + c * NC + cc);
                } else {
                    const int64_t nb = nbw & 0x7fffffff;
                    w = __ldg(gauge + (int64_t)(1 - parity) * vh * N2 + mu * gmu + nb * N2 + cc * NC + c) ^ 0x80000000u;
                }
                if (nbw < 0) w ^= tflip;
                uint8_t* bt = sB + (size_t)t * plan.b_bytes;
                const int k = h * 2 * NC + 2 * cc;
                const int n = sl * 8 + 2 * c;
                *reinterpret_cast<uint32_t*>(bt + kmajor_off(n, k, 2)) = w ^ 0x80000000u;        // (Re W, -Im W)
                *reinterpret_cast<uint32_t*>(bt + kmajor_off(n + 1, k, 2)) = __byte_perm(w, 0, 0x1032);   // (Im W, Re W)
            }
        }
        // ---- A: 4 rows (s' = 0..3) of this thread's (site, RHS), hops in two groups of 4 ----
        if (pvalid) {
            uint8_t* at = sA + (size_t)pt * plan.a_bytes;
            const uint32_t* src = in + prr;
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                uint32_t rw[4][4 * NC];
                if (g == 0) {
                    mma_rows_hop<NC, S, DAG, 0>(rw, src + nbs[0] * site_len, m);
                    mma_rows_hop<NC, S, DAG, 1>(rw, src + nbs[1] * site_len, m);
                    mma_rows_hop<NC, S, DAG, 2>(rw, src + nbs[2] * site_len, m);
                    mma_rows_hop<NC, S, DAG, 3>(rw, src + nbs[3] * site_len, m);
                } else {
                    mma_rows_hop<NC, S, DAG, 4>(rw, src + nbs[4] * site_len, m);
                    mma_rows_hop<NC, S, DAG, 5>(rw, src + nbs[5] * site_len, m);
                    mma_rows_hop<NC, S, DAG, 6>(rw, src + nbs[6] * site_len, m);
                    mma_rows_hop<NC, S, DAG, 7>(rw, src + nbs[7] * site_len, m);
                }
                // 4 N words = N chunks of 16 bytes per row; the group starts at K = 32 N g
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int n = pslot * 4 * m + s * m + prr;
#pragma unroll
                    for (int ch = 0; ch < NC; ++ch) {
                        const int k = g * 8 * NC + ch * 8;
                        *reinterpret_cast<uint4*>(at + kmajor_off(n, k, 16)) =
                            make_uint4(rw[s][4 * ch], rw[s][4 * ch + 1], rw[s][4 * ch + 2], rw[s][4 * ch + 3]);
                    }
                }
            }
        }
        // generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        fence_before_sync();
        __syncthreads();
        if (tid == 0 && !timed_out) {
            fence_after_sync();
            for (int t = 0; t < T; ++t) {
#pragma unroll
                for (int ks = 0; ks < NC; ++ks) {
                    const uint64_t ad = smem_desc(sA + (size_t)t * plan.a_bytes + ks * 2 * 16 * 128, 16 * 128, 128);
                    const uint64_t bd = smem_desc(sB + (size_t)t * plan.b_bytes + ks * 2 * 2 * 128, 2 * 128, 128);
                    mma_ss(tmem + (uint32_t)(16 * t), ad, bd, idesc, ks > 0 ? 1u : 0u);
                }
            }
            mma_commit(&sMma);
        }
        // ---- wait for the MMAs (bounded), then every thread reads its TMEM lane ----
        if (!timed_out && !mbar_wait(&sMma, phase)) {
            timed_out = true;
            sAbort = 1;
        }
        phase ^= 1u;
        fence_after_sync();
        for (int t = 0; t < T; ++t) {
            float d[16];
            tmem_ld16(tmem + lane_base + (uint32_t)(16 * t), d);
            const int64_t site = base + (int64_t)t * S_ + eslot;
            if (!row_used || site >= vh || timed_out) continue;
            S2* __restrict__ out = static_cast<S2*>(p.out);
            const S2* __restrict__ xv = static_cast<const S2*>(p.x);
            const S2* __restrict__ r0v = static_cast<const S2*>(p.r0);
            const int64_t obase = site * site_len + err_;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int64_t o = obase + (int64_t)(esp * NC + c) * m;
                const A2 v = mk2<A2>(d[eslot * 8 + 2 * c], d[eslot * 8 + 2 * c + 1]);
                if (EPI == EPI_PLAIN) {
                    out[o] = St<S>::cv(v);
                } else {
                    const A2 xx = St<S>::ld(xv[o]);
                    const float a = (float)p.a;
                    A2 res;
                    if (EPI == EPI_XPAY) {
                        res = mk2<A2>(xx.x + a * v.x, xx.y + a * v.y);
                    } else if (EPI == EPI_RESID) {
                        const A2 yy = St<S>::ld(r0v[o]);
                        res = mk2<A2>(yy.x - xx.x + a * v.x, yy.y - xx.y + a * v.y);
                    } else {
                        res = mk2<A2>(xx.x - a * v.x, xx.y - a * v.y);
                    }
                    const S2 rs = St<S>::cv(res);
                    out[o] = rs;
                    if (NV > 0) {
                        const A2 q = St<S>::ld(rs);
                        if (EPI == EPI_RESID) {
                            red[0].x += q.x * q.x + q.y * q.y;
                        } else if (EPI == EPI_SCHUR_R0) {
                            const A2 z = St<S>::ld(r0v[o]);
                            red[0].x += z.x * q.x + z.y * q.y;
                            red[0].y += z.x * q.y - z.y * q.x;
                        } else if (EPI == EPI_SCHUR_TS) {
                            red[0].x += q.x * xx.x + q.y * xx.y;
                            red[0].y += q.x * xx.y - q.y * xx.x;
                            red[NV - 1].x += q.x * q.x + q.y * q.y;
                        }
                    }
                }
            }
        }
        fence_before_sync();
        __syncthreads();
        if (sAbort) break;   // uniform: every thread read sAbort after the barrier
    }

    // every MMA of this CTA completed (or its wait gave up); free TMEM
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMmaTmemCols)
                     : "memory");
    }
    if (timed_out && err != nullptr) atomicExch(err, 1);
    if constexpr (NV > 0) {
        double2 rv[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) rv[k] = make_double2((double)red[k].x, (double)red[k].y);
        grid_reduce<NV>(rv, m, p.red);
    }
}

template <int NC, typename S>
int launch_mma(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    void (*k)(const HopParams, int*) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop_mma_kernel<NC, S, true, EPI_PLAIN> : hop_mma_kernel<NC, S, false, EPI_PLAIN>; break;
        case EPI_XPAY: k = dagger ? hop_mma_kernel<NC, S, true, EPI_XPAY> : hop_mma_kernel<NC, S, false, EPI_XPAY>; break;
        case EPI_SCHUR_R0: k = hop_mma_kernel<NC, S, false, EPI_SCHUR_R0>; break;
        case EPI_SCHUR_TS: k = hop_mma_kernel<NC, S, false, EPI_SCHUR_TS>; break;
        case EPI_SCHUR: k = hop_mma_kernel<NC, S, false, EPI_SCHUR>; break;
        case EPI_RESID: k = hop_mma_kernel<NC, S, false, EPI_RESID>; break;
        default: return set_error(QCU_ERR_INVALID, "unknown hop epilogue %d", epi);
    }
    const size_t smem = mma_smem_bytes(NC, p.m);
    static bool attr_set[2][6] = {};
    const int di = dagger ? 1 : 0;
    if (!attr_set[di][epi]) {
        QCUB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_set[di][epi] = true;
    }
    const MmaPlan plan = mma_plan(NC, p.m);
    const int64_t per_round = (int64_t)plan.T * plan.S;
    const int64_t nrounds = (p.g.vh + per_round - 1) / per_round;
    int per_sm = blocks_per_sm(reinterpret_cast<const void*>(k), kMmaThreads, smem);
    if (per_sm <= 1) {   // occupancy query unavailable: estimate from shared memory
        per_sm = (int)((220 * 1024) / (smem + 4096));
        cudaGetLastError();
    }
    const int tmem_cap = 512 / kMmaTmemCols;
    if (per_sm > tmem_cap) per_sm = tmem_cap;
    if (per_sm < 1) per_sm = 1;
    const int64_t cap = (int64_t)per_sm * sm_count();
    int grid = (int)(nrounds < cap ? nrounds : cap);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    if (grid < 1) grid = 1;
    k<<<grid, kMmaThreads, smem, st>>>(p, device_error_flag());
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace tc

// Tensor-core hop for FP16/BF16 storage: n_color 2..4 and 4*m <= 128.
// Returns QCU_ERR_UNSUPPORTED for shapes it does not cover.
bool hop_tc_supported(int nc, int m, int prec) {
    if (prec != QCU_PRECISION_HALF && prec != QCU_PRECISION_BF16) return false;
    if (nc < 2 || nc > 4) return false;   // K = 16 N, one 16-byte chunk per hop group and colour
    return 4 * m <= 128;
}

int hop_tc_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st) {
    if (!hop_tc_supported(nc, p.m, prec))
        return set_error(QCU_ERR_UNSUPPORTED, "tensor-core hop: n_color=%d m=%d precision=%d", nc, p.m, prec);
    if (p.g.vh >= (int64_t)1 << 31) return set_error(QCU_ERR_UNSUPPORTED, "half volume beyond 2^31");
    auto go = [&](auto tag) -> int {
        using S = decltype(tag);
        switch (nc) {
            case 2: return tc::launch_mma<2, S>(p, dagger, epi, st);
            case 3: return tc::launch_mma<3, S>(p, dagger, epi, st);
            default: return tc::launch_mma<4, S>(p, dagger, epi, st);
        }
    };
    if (prec == QCU_PRECISION_HALF) return go(__half{});
    return go(__nv_bfloat16{});
}

}  // namespace qcub
