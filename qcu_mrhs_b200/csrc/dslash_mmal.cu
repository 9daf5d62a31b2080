// dslash_mmal.cu -- the link-operand tensor-core hop for N <= 4 (fragment scheme in
// dslash_mmal.cuh) and the public entry points of the link-operand hop.
#include "dslash_mmal.cuh"

namespace qcub {

namespace {

// One direction for all groups of the work unit: the four neighbour words of every group
// are requested first, then each group's two projections and one MMA that adds the forward
// and backward hop into the direction class's FP32 accumulator quad through the MMA's C
// operand (Q[n] is the x/y quad or the z/t quad of group n).
template <typename S, int MU, int SF, int NTC, bool EXACT>
__device__ __forceinline__ void mmal_dir(float (&Q)[NTC][4], const uint32_t* __restrict__ pf,
                                         const uint32_t* __restrict__ qf, const uint32_t* __restrict__ pb,
                                         const uint32_t* __restrict__ qb, const uint32_t (&A)[4], uint32_t lmf,
                                         uint32_t lmb, int rb0, int q, int m) {
    using M = LMma<S>;
    constexpr int SB = -SF;
    uint32_t w[NTC][4];
#pragma unroll
    for (int n = 0; n < NTC; ++n) {
        if (!EXACT && rb0 + 4 * n >= m) break;   // warp-uniform
        int d = 4 * n;
        if (!EXACT) d += min(0, m - 1 - (rb0 + 4 * n + q));   // last partial group: clamp the RHS
        w[n][0] = __ldg(pf + d);
        w[n][1] = __ldg(qf + d);
        w[n][2] = __ldg(pb + d);
        w[n][3] = __ldg(qb + d);
    }
#pragma unroll
    for (int n = 0; n < NTC; ++n) {
        if (!EXACT && rb0 + 4 * n >= m) break;
        const uint32_t hf = lproject<S, MU, SF>(w[n][0], w[n][1], lmf);
        const uint32_t hb = lproject<S, MU, SB>(w[n][2], w[n][3], lmb);
        M::mma(Q[n], A, hf, hb, Q[n][0], Q[n][1], Q[n][2], Q[n][3]);
    }
}

// Resident blocks per SM asked of the register allocator: 3 (80 registers) for the forms
// without a reduction, 2 for the reducing forms (their epilogue words and partial sums
// would spill at 80).
template <int EPI> struct LMinBlocks {
    static constexpr int value = (EPI == EPI_SCHUR_R0 || EPI == EPI_SCHUR_TS || EPI == EPI_RESID) ? 2 : 3;
};

template <typename S, int NC, bool DAG, int EPI, int NTC, bool EXACT, bool PRE>
__global__ void __launch_bounds__(kLThreads, LMinBlocks<EPI>::value) hop_mmal_kernel(const HopParams p, int nchunk) {
    using M = LMma<S>;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int NVR = NV > 0 ? NV : 1;
    constexpr int NY = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : 0;   // reads r0 / y
    constexpr uint32_t N2 = NC * NC;
    constexpr int SF = DAG ? 1 : -1;   // forward projector 1 - s g: sign of gamma
    static_assert(NC >= 2 && NC <= 4, "one M tile holds the sum and diff rows for N <= 4");
    if (skip_launch(p.done, p.gate)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3, hh = g & 1, q = g >> 1;
    const int cls = g >> 2, cc = g & 3;          // D/A rows of this lane: class, colour
    const int m = p.m;
    const uint32_t SW = 4u * NC * (uint32_t)m;   // 32-bit words per site
    const int ccl = min(cc, NC - 1), ct = min(t, NC - 1);
    const uint32_t okm = (cc < NC && t < NC) ? 0xffffffffu : 0u;   // this lane's A entries exist
    const bool sok = cc < NC;                    // this lane's output colour exists
    // input shifted to the lane's B column RHS (q of a group); the lane pointers to the words
    // p_h, q of the projections follow once the chunk is known
    const uint32_t* __restrict__ in = static_cast<const uint32_t*>(p.in) + q;
    // output words of this lane: spins 2 cls, 2 cls + 1 of colour g % 4, RHS t of a group
    const uint32_t os = (uint32_t)((2 * cls * NC + ccl) * m + t);
    const uint32_t osn = (uint32_t)(NC * m);
    // lane projection multipliers of MU 1 and MU 2 (forward / backward)
    const uint32_t m1f = hh ? unit_pair<S>(SF, SF) : unit_pair<S>(-SF, -SF);
    const uint32_t m2f = hh ? unit_pair<S>(SF, -SF) : unit_pair<S>(-SF, SF);
    const uint32_t m1b = m1f ^ 0x80008000u, m2b = m2f ^ 0x80008000u;
    // diff-row phases per direction, and the lane sign that flips spin 3 between the two
    // directions of a class (diff lanes only)
    const LPhase ph0 = lphase_lane<LRecon<0, SF>::C2>(cls != 0);
    const LPhase ph1 = lphase_lane<LRecon<1, SF>::C2>(cls != 0);
    const LPhase ph2 = lphase_lane<LRecon<2, SF>::C2>(cls != 0);
    const LPhase ph3 = lphase_lane<LRecon<3, SF>::C2>(cls != 0);
    const float fl = cls ? -1.f : 1.f;

    const uint32_t vh = (uint32_t)p.g.vh;
    const int parity = p.parity;
    const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
    uint32_t* __restrict__ out = static_cast<uint32_t*>(p.out);
    const uint32_t* __restrict__ xv = static_cast<const uint32_t*>(p.x);
    const uint32_t* __restrict__ yv = static_cast<const uint32_t*>(p.r0);
    const uint32_t gblk = vh * N2;   // words of one (mu, parity) block of the gauge
    const uint32_t* __restrict__ glf = gauge + (size_t)parity * gblk + (uint32_t)(ccl * NC + ct);
    const uint32_t* __restrict__ glb = gauge + (size_t)(1 - parity) * gblk + (uint32_t)(ct * NC + ccl);
    const size_t gmu = 2 * (size_t)gblk;
    const uint32_t tflip = p.t_sign < 0 ? 0x80008000u : 0u;
    const uint32_t lxh = (uint32_t)p.g.lxh, Ly = (uint32_t)p.g.L[1], Lz = (uint32_t)p.g.L[2],
                   Lt = (uint32_t)p.g.L[3];
    const uint32_t sy = lxh, sz = lxh * Ly, st = sz * Lz;

    // work units: warp gw takes chunk gw % nchunk of the sites gw / nchunk + k stride
    const int64_t gw = (int64_t)blockIdx.x * kLWarps + warp;
    const int64_t nw = (int64_t)gridDim.x * kLWarps;
    const int chunk = (int)(gw % nchunk);
    const uint32_t site_stride = (uint32_t)(nw / nchunk);
    const uint32_t site0 = gw < (int64_t)site_stride * nchunk ? (uint32_t)(gw / nchunk) : vh;
    const int rb0 = chunk * NTC * 4;
    // groups with a live RHS (per-RHS activity flags); the others are loaded and computed
    // like the rest (no per-group branches between the loads) but not stored
    const uint32_t gmask = active_groups<NTC>(p.active, rb0, m);
    const uint32_t* __restrict__ inA = in + rb0 + (hh * NC + ct) * m;
    const uint32_t* __restrict__ inB01 = in + rb0 + ((3 - hh) * NC + ct) * m;
    const uint32_t* __restrict__ inB23 = in + rb0 + ((2 + hh) * NC + ct) * m;

    float2 red[NTC][NVR];
#pragma unroll
    for (int n = 0; n < NTC; ++n)
#pragma unroll
        for (int k = 0; k < NVR; ++k) red[n][k] = make_float2(0.f, 0.f);

    for (uint32_t site = site0; site < vh; site += site_stride) {
        // neighbours and the lane's link words W_f[g%4][t], W_b[g%4][t] of the 4 directions
        uint32_t nb0, nb1, nb2, nb3, nb4, nb5, nb6, nb7;
        uint32_t wf[4], wb[4];
        if constexpr (PRE) {
            const uint4* nt = reinterpret_cast<const uint4*>(p.nbr) + ((size_t)parity * vh + site) * 2;
            const uint4 na = __ldg(nt), nc4 = __ldg(nt + 1);
            nb0 = na.x; nb1 = na.y; nb2 = na.z; nb3 = na.w;
            nb4 = nc4.x; nb5 = nc4.y; nb6 = nc4.z; nb7 = nc4.w;
            const uint32_t* lk = static_cast<const uint32_t*>(p.links) + ((size_t)parity * vh + site) * 8 * N2 +
                                 (uint32_t)(ccl * NC + ct);
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                wf[mu] = __ldg(lk + 2 * mu * N2);
                wb[mu] = __ldg(lk + (2 * mu + 1) * N2);
            }
        } else {
            const SiteXYZT c = site_coords(p.g, site);
            const uint32_t xh = (uint32_t)c.xh;
            const int xodd = (parity ^ (c.y + c.z + c.t)) & 1;
            const uint32_t row = site - xh;
            nb0 = row + (xodd ? (xh + 1 == lxh ? 0u : xh + 1) : xh);
            nb1 = row + (xodd ? xh : (xh == 0 ? lxh - 1 : xh - 1));
            nb2 = site + sy - ((uint32_t)c.y + 1 == Ly ? Ly * sy : 0u);
            nb3 = site - sy + ((uint32_t)c.y == 0 ? Ly * sy : 0u);
            nb4 = site + sz - ((uint32_t)c.z + 1 == Lz ? Lz * sz : 0u);
            nb5 = site - sz + ((uint32_t)c.z == 0 ? Lz * sz : 0u);
            const bool wf_t = ((uint32_t)c.t + 1 == Lt), wb_t = (c.t == 0);
            nb6 = site + st - (wf_t ? Lt * st : 0u);
            nb7 = site - st + (wb_t ? Lt * st : 0u);
            const uint32_t nbb[4] = {nb1, nb3, nb5, nb7};
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                wf[mu] = __ldg(glf + mu * gmu + (size_t)site * N2);
                wb[mu] = __ldg(glb + mu * gmu + (size_t)nbb[mu] * N2) ^ 0x80000000u;   // conj
            }
            if (wf_t) wf[3] ^= tflip;   // t-boundary sign
            if (wb_t) wb[3] ^= tflip;
        }
        const size_t sbase = (size_t)site * SW + rb0;

        // epilogue operands of this site, requested first
        uint32_t xw[NTC][2], yw[NTC][2];
        if constexpr (EPI != EPI_PLAIN) {
#pragma unroll
            for (int n = 0; n < NTC; ++n) {
                xw[n][0] = xw[n][1] = yw[n][0] = yw[n][1] = 0u;
                if (!EXACT && rb0 + 4 * n >= m) break;
                if (sok && (EXACT || rb0 + 4 * n + t < m)) {
                    const size_t o = sbase + os + 4 * n;
                    xw[n][0] = __ldg(xv + o);
                    xw[n][1] = __ldg(xv + o + osn);
                    if (NY) {
                        yw[n][0] = __ldg(yv + o);
                        yw[n][1] = __ldg(yv + o + osn);
                    }
                }
            }
        }

        float Qxy[NTC][4], Qzt[NTC][4];
#pragma unroll
        for (int n = 0; n < NTC; ++n)
#pragma unroll
            for (int k = 0; k < 4; ++k) Qxy[n][k] = Qzt[n][k] = 0.f;
        uint32_t A[4];
        // y, then spin 3 (diff column h0, registers 0 and 2) negated, then x: spin 3 takes
        // x - y (the y projector's spin-3 phase is minus its diff-row phase)
        mmal_a(A, wf[1], wb[1], okm, ph1.sel, ph1.mf, ph1.mb);
        mmal_dir<S, 1, SF, NTC, EXACT>(Qxy, inA + (size_t)nb2 * SW, inB01 + (size_t)nb2 * SW, inA + (size_t)nb3 * SW,
                                       inB01 + (size_t)nb3 * SW, A, m1f, m1b, rb0, q, m);
#pragma unroll
        for (int n = 0; n < NTC; ++n) {
            Qxy[n][0] *= fl;
            Qxy[n][2] *= fl;
        }
        mmal_a(A, wf[0], wb[0], okm, ph0.sel, ph0.mf, ph0.mb);
        mmal_dir<S, 0, SF, NTC, EXACT>(Qxy, inA + (size_t)nb0 * SW, inB01 + (size_t)nb0 * SW, inA + (size_t)nb1 * SW,
                                       inB01 + (size_t)nb1 * SW, A, 0u, 0u, rb0, q, m);
        // z, then spin 3 (diff column h1, registers 1 and 3) negated, then t (boundary sign
        // folded into the links)
        mmal_a(A, wf[2], wb[2], okm, ph2.sel, ph2.mf, ph2.mb);
        mmal_dir<S, 2, SF, NTC, EXACT>(Qzt, inA + (size_t)nb4 * SW, inB23 + (size_t)nb4 * SW, inA + (size_t)nb5 * SW,
                                       inB23 + (size_t)nb5 * SW, A, m2f, m2b, rb0, q, m);
#pragma unroll
        for (int n = 0; n < NTC; ++n) {
            Qzt[n][1] *= fl;
            Qzt[n][3] *= fl;
        }
        mmal_a(A, wf[3], wb[3], okm, ph3.sel, ph3.mf, ph3.mb);
        mmal_dir<S, 3, SF, NTC, EXACT>(Qzt, inA + (size_t)nb6 * SW, inB23 + (size_t)nb6 * SW, inA + (size_t)nb7 * SW,
                                       inB23 + (size_t)nb7 * SW, A, 0u, 0u, rb0, q, m);

#pragma unroll
        for (int n = 0; n < NTC; ++n) {
            if (!EXACT && rb0 + 4 * n >= m) break;   // warp-uniform
            const bool rok = sok && (EXACT || rb0 + 4 * n + t < m);
            const size_t o = sbase + os + 4 * n;
            // the lane's two spins (2 cls, 2 cls + 1) of (colour g % 4, RHS t): sum lanes take
            // both quads as they are; diff lanes take the x/y quad's columns crosswise (the
            // x and y projectors exchange the half spinors)
            float2 ov[2];
            ov[0].x = Qzt[n][0] + (cls ? Qxy[n][1] : Qxy[n][0]);
            ov[0].y = Qzt[n][2] + (cls ? Qxy[n][3] : Qxy[n][2]);
            ov[1].x = Qzt[n][1] + (cls ? Qxy[n][0] : Qxy[n][1]);
            ov[1].y = Qzt[n][3] + (cls ? Qxy[n][2] : Qxy[n][3]);
            if (!rok || !((gmask >> n) & 1u)) continue;
            if constexpr (EPI == EPI_PLAIN) {
                out[o] = M::pack(ov[0].x, ov[0].y);
                out[o + osn] = M::pack(ov[1].x, ov[1].y);
            } else {
                const float a = (float)p.a;
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const float2 xx = M::unpack(xw[n][k]);
                    float2 res;
                    if (EPI == EPI_XPAY) {
                        res = make_float2(xx.x + a * ov[k].x, xx.y + a * ov[k].y);
                    } else if (EPI == EPI_RESID) {
                        const float2 yy = M::unpack(yw[n][k]);
                        res = make_float2(yy.x - xx.x + a * ov[k].x, yy.y - xx.y + a * ov[k].y);
                    } else {
                        res = make_float2(xx.x - a * ov[k].x, xx.y - a * ov[k].y);
                    }
                    const uint32_t rs = M::pack(res.x, res.y);
                    out[o + (k ? osn : 0u)] = rs;
                    if constexpr (NV > 0) {
                        const float2 rr = M::unpack(rs);
                        if (EPI == EPI_RESID) {
                            red[n][0].x += rr.x * rr.x + rr.y * rr.y;
                        } else if (EPI == EPI_SCHUR_R0) {   // <r0, out> = sum conj(r0) out
                            const float2 qq = M::unpack(yw[n][k]);
                            red[n][0].x += qq.x * rr.x + qq.y * rr.y;
                            red[n][0].y += qq.x * rr.y - qq.y * rr.x;
                        } else if (EPI == EPI_SCHUR_TS) {  // <out, x>, <out, out>
                            red[n][0].x += rr.x * xx.x + rr.y * xx.y;
                            red[n][0].y += rr.x * xx.y - rr.y * xx.x;
                            red[n][NV - 1].x += rr.x * rr.x + rr.y * rr.y;
                        }
                    }
                }
            }
        }
    }
    if constexpr (NV > 0) {
        // lanes (g, t) hold RHS rb0 + 4n + t: sum over g (fixed butterfly), then over the
        // block's warps of the same chunk in order, then the common grid stage
        __shared__ double2 wsum[kLWarps][NV][kLMaxChunkRhs];
        __shared__ double2 bsum[NV * kMaxRhs];
#pragma unroll
        for (int n = 0; n < NTC; ++n)
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                double vx = (double)red[n][k].x, vy = (double)red[n][k].y;
#pragma unroll
                for (int off = 4; off < 32; off <<= 1) {
                    vx += __shfl_xor_sync(0xffffffffu, vx, off);
                    vy += __shfl_xor_sync(0xffffffffu, vy, off);
                }
                if (g == 0) wsum[warp][k][4 * n + t] = make_double2(vx, vy);
            }
        __syncthreads();
        for (int idx = threadIdx.x; idx < NV * m; idx += blockDim.x) {
            const int k = idx / m, rhs = idx - k * m;
            const int ch = rhs / (4 * NTC), loc = rhs - ch * 4 * NTC;
            double2 s = make_double2(0.0, 0.0);
            for (int w = 0; w < kLWarps; ++w) {
                if ((int)(((int64_t)blockIdx.x * kLWarps + w) % nchunk) != ch) continue;
                s.x += wsum[w][k][loc].x;
                s.y += wsum[w][k][loc].y;
            }
            bsum[idx] = s;
        }
        __syncthreads();
        publish_and_finish<NV>(bsum, m, p.red);
    }
}

// ---------------------------------------------------------------------------------
// Staged variant (the solver's hops: per-site tables present, m = 4, 8, 12 or 16).
// Each warp keeps two shared-memory stages.  A stage holds the 8 neighbour site blocks
// (16 N m bytes each, contiguous in the gathered layout), the site's hop-link block
// (8 N^2 words) and, for the epilogues that read them, the site's x and r0 blocks.  While
// the warp computes one site from one stage, the bulk-copy engine (cp.async.bulk, no
// multicast) fills the other stage for the warp's next site: lanes 0-7 each copy one
// neighbour block, lane 8 the links, lanes 9 and 10 x and r0; completion is counted in
// bytes on the stage's mbarrier.  Fragment words are then read from shared memory at
// compile-time offsets.  Every mbarrier wait is bounded: a wait that gives up sets the
// device error flag, the warp drains its copies still in flight (again bounded) and skips
// its remaining sites, so a broken pipeline ends the kernel with an error, never a hang.
constexpr int kTWarps = 4;
constexpr int kTThreads = kTWarps * 32;
constexpr int kTStages = 2;
constexpr int kTBarBytes = 64;   // mbarriers of the block (kTWarps x kTStages x 8 bytes)

__device__ __forceinline__ uint32_t lsmem(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool lbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: the clock is read only once the first try has failed (in the common case
// the copies have landed and the wait costs one try); gives up after `limit` cycles
__device__ __forceinline__ bool lbar_wait(uint32_t bar, uint32_t parity, long long limit) {
    if (lbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (lbar_try(bar, parity)) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// Bytes of one stage: 8 neighbour blocks, the link block, NX epilogue blocks.
__host__ __device__ constexpr int tstage_bytes(int nc, int m, int nx) { return (8 + nx) * 16 * nc * m + 32 * nc * nc; }

// One direction of the staged kernel for NT tiles: tile n takes the group of 4 RHS at word
// offset go(n) of a spin-colour row (4 n when all groups are live, DENSE).
template <typename S, int MU, int SF, int NT, bool DENSE>
__device__ __forceinline__ void mmal_dir_s(float (&Q)[NT][4], const uint32_t* pf, const uint32_t* qf,
                                           const uint32_t* pb, const uint32_t* qb, const uint32_t (&A)[4],
                                           uint32_t lmf, uint32_t lmb, const int (&go)[NT]) {
    using M = LMma<S>;
    constexpr int SB = -SF;
    uint32_t w[NT][4];
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        const int o = DENSE ? 4 * n : go[n];
        w[n][0] = pf[o];
        w[n][1] = qf[o];
        w[n][2] = pb[o];
        w[n][3] = qb[o];
    }
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        const uint32_t hf = lproject<S, MU, SF>(w[n][0], w[n][1], lmf);
        const uint32_t hb = lproject<S, MU, SB>(w[n][2], w[n][3], lmb);
        M::mma(Q[n], A, hf, hb, Q[n][0], Q[n][1], Q[n][2], Q[n][3]);
    }
}

template <typename S, int NC, bool DAG, int EPI, int NTC>
__global__ void __launch_bounds__(kTThreads) hop_mmal_tma_kernel(const HopParams p, int* err) {
    using M = LMma<S>;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int NVR = NV > 0 ? NV : 1;
    constexpr int NX = EPI == EPI_PLAIN ? 0 : ((EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 2 : 1);
    constexpr int MR = 4 * NTC;                  // RHS count
    constexpr uint32_t N2 = NC * NC;
    constexpr int SW = 4 * NC * MR;              // words of a site block
    constexpr int SBY = 4 * SW;                  // its bytes
    constexpr int LW = 8 * NC * NC;              // words of a link block
    constexpr int STW = tstage_bytes(NC, MR, NX) / 4;
    constexpr uint32_t TX = (uint32_t)tstage_bytes(NC, MR, NX);
    constexpr int SF = DAG ? 1 : -1;
    static_assert(NC >= 2 && NC <= 4 && MR <= 16, "staged hop: N <= 4, m <= 16");
    extern __shared__ __align__(16) unsigned char tsm[];
    if (skip_launch(p.done, p.gate)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3, hh = g & 1, q = g >> 1;
    const int cls = g >> 2, cc = g & 3;
    const int ccl = min(cc, NC - 1), ct = min(t, NC - 1);
    const uint32_t okm = (cc < NC && t < NC) ? 0xffffffffu : 0u;
    const bool sok = cc < NC;
    const int oa = (hh * NC + ct) * MR + q;
    const int ob01 = ((3 - hh) * NC + ct) * MR + q;
    const int ob23 = ((2 + hh) * NC + ct) * MR + q;
    const int os = (2 * cls * NC + ccl) * MR + t;
    constexpr int osn = NC * MR;
    const int lo = ccl * NC + ct;                // the lane's element of a link matrix
    const uint32_t m1f = hh ? unit_pair<S>(SF, SF) : unit_pair<S>(-SF, -SF);
    const uint32_t m2f = hh ? unit_pair<S>(SF, -SF) : unit_pair<S>(-SF, SF);
    const uint32_t m1b = m1f ^ 0x80008000u, m2b = m2f ^ 0x80008000u;
    const LPhase ph0 = lphase_lane<LRecon<0, SF>::C2>(cls != 0);
    const LPhase ph1 = lphase_lane<LRecon<1, SF>::C2>(cls != 0);
    const LPhase ph2 = lphase_lane<LRecon<2, SF>::C2>(cls != 0);
    const LPhase ph3 = lphase_lane<LRecon<3, SF>::C2>(cls != 0);
    const float fl = cls ? -1.f : 1.f;
    const uint32_t gmask = active_groups<NTC>(p.active, 0, MR);

    const uint32_t vh = (uint32_t)p.g.vh;
    const int parity = p.parity;
    const unsigned char* __restrict__ in = static_cast<const unsigned char*>(p.in);
    const unsigned char* __restrict__ links = static_cast<const unsigned char*>(p.links);
    const unsigned char* __restrict__ xv = static_cast<const unsigned char*>(p.x);
    const unsigned char* __restrict__ yv = static_cast<const unsigned char*>(p.r0);
    const uint32_t* __restrict__ nbr = p.nbr + (size_t)parity * vh * 8;
    uint32_t* __restrict__ out = static_cast<uint32_t*>(p.out);

    // this warp's stages and barriers
    uint32_t* stage = reinterpret_cast<uint32_t*>(tsm + kTBarBytes) + (size_t)warp * kTStages * STW;
    const uint32_t bar0 = lsmem(tsm) + 8 * (warp * kTStages);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < kTStages; ++k)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8 * k) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();

    const uint32_t gw = blockIdx.x * kTWarps + warp;
    const uint32_t nw = gridDim.x * kTWarps;
    // copy the blocks of `site` into stage k (lane 0 arms the barrier with the byte count;
    // lanes 0-7 take neighbour nbi, lane 8 the links, lanes 9-10 the epilogue blocks)
    // lane roles of a copy round, fixed for the kernel: source base and per-site stride,
    // destination offset in the stage, bytes; the copy itself is predicated, not branched
    // (wait self-test: the barrier is armed, no copy is issued, every wait runs out)
    const bool cp_nb = lane < 8, cp_on = lane < 9 + NX && !p.wait_test;
    const long long wlim = p.wait_limit > 0 ? p.wait_limit : (1ll << 31);   // about a second
    const uint32_t cp_flight = p.wait_test ? 0u : 1u;   // 1: a stage's copies are in flight
    const unsigned char* cp_base = lane == 8 ? links + (size_t)parity * vh * (LW * 4)
                                 : (lane == 9 ? xv : (lane == 10 ? yv : in));
    const uint32_t cp_stride = lane == 8 ? LW * 4 : SBY;
    const uint32_t cp_dst = lane < 8 ? lane * SBY : (lane == 8 ? 8 * SBY : 8 * SBY + LW * 4 + (lane - 9) * SBY);
    const uint32_t cp_bytes = lane == 8 ? LW * 4 : SBY;
    const uint32_t stage_s = lsmem(stage);
    auto issue = [&](int k, uint32_t site, uint32_t nbi) {
        const uint32_t bar = bar0 + 8 * k;
        if (lane == 0) asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(TX) : "memory");
        __syncwarp();
        const unsigned char* src = cp_base + (size_t)(cp_nb ? nbi : site) * cp_stride;
        const uint32_t dst = stage_s + k * (STW * 4) + cp_dst;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %4, 0;\n\t"
            "@p fence.proxy.async.shared::cta;\n\t"
            "@p cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n\t}"
            ::"r"(dst), "l"(src), "r"(cp_bytes), "r"(bar), "r"((uint32_t)cp_on) : "memory");
    };

    float2 red[NTC][NVR];
#pragma unroll
    for (int n = 0; n < NTC; ++n)
#pragma unroll
        for (int k = 0; k < NVR; ++k) red[n][k] = make_float2(0.f, 0.f);

    // Live groups: the warp computes NA = popcount(gmask) tiles, tile n on the n-th live
    // group (groups in order).  Each NA is compiled separately, so every form is
    // straight-line code and the all-live form (NA = NTC) has compile-time offsets.
    const int na = __popc(gmask);
    auto sites = [&](auto na_tag) {
        constexpr int NA = decltype(na_tag)::value;
        constexpr bool DENSE = NA == NTC;
        int go[NA];   // word offset of tile n's group: the n-th set bit of gmask, times 4
        uint32_t rest = gmask;
#pragma unroll
        for (int n = 0; n < NA; ++n) {
            go[n] = 4 * (__ffs(rest) - 1);
            rest &= rest - 1u;
        }
        float2 rt[NA][NVR];   // this form's partial sums per tile
#pragma unroll
        for (int n = 0; n < NA; ++n)
#pragma unroll
            for (int kk = 0; kk < NVR; ++kk) rt[n][kk] = make_float2(0.f, 0.f);
        uint32_t site = gw;
        uint32_t inflight = 0;   // bit k: stage k has copies in flight
        uint32_t use = 0;        // uses of each stage so far (bit k = parity of stage k's next wait)
        if (site < vh) {
            issue(0, site, lane < 8 ? __ldg(nbr + (size_t)site * 8 + lane) : 0u);
            inflight |= cp_flight;
        }
        // neighbour index of the next site, loaded one site ahead
        uint32_t nb_next = (site + nw < vh && lane < 8) ? __ldg(nbr + (size_t)(site + nw) * 8 + lane) : 0u;
        bool ok = true;
        for (int it = 0; site < vh; ++it, site += nw) {
            const int k = it & 1;
            const uint32_t nxt = site + nw;
            if (nxt < vh) {   // the other stage was released by the previous site's __syncwarp
                issue(k ^ 1, nxt, nb_next);
                inflight |= cp_flight << (k ^ 1);
                nb_next = (nxt + nw < vh && lane < 8) ? __ldg(nbr + (size_t)(nxt + nw) * 8 + lane) : 0u;
            }
            if (!lbar_wait(bar0 + 8 * k, (use >> k) & 1u, wlim)) {
                ok = false;
                break;
            }
            use ^= 1u << k;
            inflight &= ~(1u << k);
            const uint32_t* sb = stage + k * STW;       // neighbour blocks
            const uint32_t* lk = sb + 8 * SW + lo;      // links
            const uint32_t* ep = sb + 8 * SW + LW + os; // x, then r0
            float Qxy[NA][4], Qzt[NA][4];
#pragma unroll
            for (int n = 0; n < NA; ++n)
#pragma unroll
                for (int e = 0; e < 4; ++e) Qxy[n][e] = Qzt[n][e] = 0.f;
            uint32_t A[4];
            mmal_a(A, lk[2 * N2], lk[3 * N2], okm, ph1.sel, ph1.mf, ph1.mb);
            mmal_dir_s<S, 1, SF, NA, DENSE>(Qxy, sb + 2 * SW + oa, sb + 2 * SW + ob01, sb + 3 * SW + oa, sb + 3 * SW + ob01, A,
                                      m1f, m1b, go);
#pragma unroll
            for (int n = 0; n < NA; ++n) {
                Qxy[n][0] *= fl;
                Qxy[n][2] *= fl;
            }
            mmal_a(A, lk[0], lk[N2], okm, ph0.sel, ph0.mf, ph0.mb);
            mmal_dir_s<S, 0, SF, NA, DENSE>(Qxy, sb + oa, sb + ob01, sb + SW + oa, sb + SW + ob01, A, 0u, 0u, go);
            mmal_a(A, lk[4 * N2], lk[5 * N2], okm, ph2.sel, ph2.mf, ph2.mb);
            mmal_dir_s<S, 2, SF, NA, DENSE>(Qzt, sb + 4 * SW + oa, sb + 4 * SW + ob23, sb + 5 * SW + oa, sb + 5 * SW + ob23, A,
                                      m2f, m2b, go);
#pragma unroll
            for (int n = 0; n < NA; ++n) {
                Qzt[n][1] *= fl;
                Qzt[n][3] *= fl;
            }
            mmal_a(A, lk[6 * N2], lk[7 * N2], okm, ph3.sel, ph3.mf, ph3.mb);
            mmal_dir_s<S, 3, SF, NA, DENSE>(Qzt, sb + 6 * SW + oa, sb + 6 * SW + ob23, sb + 7 * SW + oa, sb + 7 * SW + ob23, A,
                                      0u, 0u, go);
            const size_t ob = (size_t)site * SW + os;
#pragma unroll
            for (int n = 0; n < NA; ++n) {
                const int gn = DENSE ? 4 * n : go[n];   // word offset of the tile's group
                float2 ov[2];
                ov[0].x = Qzt[n][0] + (cls ? Qxy[n][1] : Qxy[n][0]);
                ov[0].y = Qzt[n][2] + (cls ? Qxy[n][3] : Qxy[n][2]);
                ov[1].x = Qzt[n][1] + (cls ? Qxy[n][0] : Qxy[n][1]);
                ov[1].y = Qzt[n][3] + (cls ? Qxy[n][2] : Qxy[n][3]);
                if constexpr (EPI == EPI_PLAIN) {
                    const uint32_t w0 = M::pack(ov[0].x, ov[0].y), w1 = M::pack(ov[1].x, ov[1].y);
                    if (sok) {
                        out[ob + gn] = w0;
                        out[ob + gn + osn] = w1;
                    }
                } else if (sok) {
                    const float a = (float)p.a;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const uint32_t xw = ep[gn + (e ? osn : 0)];
                        const float2 xx = M::unpack(xw);
                        float2 res;
                        if (EPI == EPI_XPAY) {
                            res = make_float2(xx.x + a * ov[e].x, xx.y + a * ov[e].y);
                        } else if (EPI == EPI_RESID) {
                            const float2 yy = M::unpack(ep[SW + gn + (e ? osn : 0)]);
                            res = make_float2(yy.x - xx.x + a * ov[e].x, yy.y - xx.y + a * ov[e].y);
                        } else {
                            res = make_float2(xx.x - a * ov[e].x, xx.y - a * ov[e].y);
                        }
                        const uint32_t rs = M::pack(res.x, res.y);
                        out[ob + gn + (e ? osn : 0)] = rs;
                        if constexpr (NV > 0) {
                            const float2 rr = M::unpack(rs);
                            if (EPI == EPI_RESID) {
                                rt[n][0].x += rr.x * rr.x + rr.y * rr.y;
                            } else if (EPI == EPI_SCHUR_R0) {   // <r0, out> = sum conj(r0) out
                                const float2 qq = M::unpack(ep[SW + gn + (e ? osn : 0)]);
                                rt[n][0].x += qq.x * rr.x + qq.y * rr.y;
                                rt[n][0].y += qq.x * rr.y - qq.y * rr.x;
                            } else if (EPI == EPI_SCHUR_TS) {  // <out, x>, <out, out>
                                rt[n][0].x += rr.x * xx.x + rr.y * xx.y;
                                rt[n][0].y += rr.x * xx.y - rr.y * xx.x;
                                rt[n][NV - 1].x += rr.x * rr.x + rr.y * rr.y;
                            }
                        }
                    }
                }
            }
            __syncwarp();   // every lane has read stage k before it is refilled
        }
        if (!ok) {
            // a wait gave up: record it and let the copies still in flight land (bounded)
            if (lane == 0) atomicExch(err, 1);
            for (int k = 0; k < kTStages; ++k)
                if ((inflight >> k) & 1u) {
                    if (!lbar_wait(bar0 + 8 * k, (use >> k) & 1u, wlim)) break;
                }
        }
        // partial sums back to their groups
#pragma unroll
        for (int n = 0; n < NA; ++n)
#pragma unroll
            for (int gi = 0; gi < NTC; ++gi)
                if ((DENSE ? 4 * n : go[n]) == 4 * gi)
#pragma unroll
                    for (int kk = 0; kk < NVR; ++kk) {
                        red[gi][kk].x += rt[n][kk].x;
                        red[gi][kk].y += rt[n][kk].y;
                    }
    };
    if (na == NTC) {
        sites(std::integral_constant<int, NTC>{});
    } else if (na == 1) {
        if constexpr (NTC > 1) sites(std::integral_constant<int, 1>{});
    } else if (na == 2) {
        if constexpr (NTC > 2) sites(std::integral_constant<int, 2>{});
    } else if (na == 3) {
        if constexpr (NTC > 3) sites(std::integral_constant<int, 3>{});
    }   // na == 0: nothing to compute, the outputs stay as they were

    if constexpr (NV > 0) {
        __shared__ double2 wsum[kTWarps][NV][kLMaxChunkRhs];
        __shared__ double2 bsum[NV * kMaxRhs];
#pragma unroll
        for (int n = 0; n < NTC; ++n)
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                double vx = (double)red[n][k].x, vy = (double)red[n][k].y;
#pragma unroll
                for (int off = 4; off < 32; off <<= 1) {
                    vx += __shfl_xor_sync(0xffffffffu, vx, off);
                    vy += __shfl_xor_sync(0xffffffffu, vy, off);
                }
                if (g == 0) wsum[warp][k][4 * n + t] = make_double2(vx, vy);
            }
        __syncthreads();
        for (int idx = threadIdx.x; idx < NV * MR; idx += blockDim.x) {
            const int k = idx / MR, rhs = idx - k * MR;
            double2 s = make_double2(0.0, 0.0);
            for (int w = 0; w < kTWarps; ++w) {
                s.x += wsum[w][k][rhs].x;
                s.y += wsum[w][k][rhs].y;
            }
            bsum[idx] = s;
        }
        __syncthreads();
        publish_and_finish<NV>(bsum, MR, p.red);
    }
}

template <typename S, int NC, int NTC, int EPI, bool DAG>
void* tma_kernel_ptr() {
    return reinterpret_cast<void*>(hop_mmal_tma_kernel<S, NC, DAG, EPI, NTC>);
}

template <typename S, int NC, int NTC>
int launch_mmal_tma(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    void (*k)(const HopParams, int*) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop_mmal_tma_kernel<S, NC, true, EPI_PLAIN, NTC> : hop_mmal_tma_kernel<S, NC, false, EPI_PLAIN, NTC>; break;
        case EPI_XPAY: k = dagger ? hop_mmal_tma_kernel<S, NC, true, EPI_XPAY, NTC> : hop_mmal_tma_kernel<S, NC, false, EPI_XPAY, NTC>; break;
        case EPI_SCHUR_R0: k = hop_mmal_tma_kernel<S, NC, false, EPI_SCHUR_R0, NTC>; break;
        case EPI_SCHUR_TS: k = hop_mmal_tma_kernel<S, NC, false, EPI_SCHUR_TS, NTC>; break;
        case EPI_SCHUR: k = hop_mmal_tma_kernel<S, NC, false, EPI_SCHUR, NTC>; break;
        case EPI_RESID: k = hop_mmal_tma_kernel<S, NC, false, EPI_RESID, NTC>; break;
        default: return set_error(QCU_ERR_INVALID, "epilogue %d", epi);
    }
    const int nx = epi == EPI_PLAIN ? 0 : ((epi == EPI_SCHUR_R0 || epi == EPI_RESID) ? 2 : 1);
    const size_t smem = kTBarBytes + (size_t)kTWarps * kTStages * tstage_bytes(NC, 4 * NTC, nx);
    int* err = device_error_flag();
    if (!err) return set_error(QCU_ERR_CUDA, "device error flag unavailable");
    int grid = resident_grid(k, kTThreads, p.g.vh * 32, smem);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    k<<<grid, kTThreads, smem, st>>>(p, err);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <typename S, int NC, int NTC, bool EXACT, bool PRE>
int launch_mmal_t(const HopParams& p, bool dagger, int epi, int nchunk, cudaStream_t st) {
    void (*k)(const HopParams, int) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop_mmal_kernel<S, NC, true, EPI_PLAIN, NTC, EXACT, PRE> : hop_mmal_kernel<S, NC, false, EPI_PLAIN, NTC, EXACT, PRE>; break;
        case EPI_XPAY: k = dagger ? hop_mmal_kernel<S, NC, true, EPI_XPAY, NTC, EXACT, PRE> : hop_mmal_kernel<S, NC, false, EPI_XPAY, NTC, EXACT, PRE>; break;
        case EPI_SCHUR_R0: k = hop_mmal_kernel<S, NC, false, EPI_SCHUR_R0, NTC, EXACT, PRE>; break;
        case EPI_SCHUR_TS: k = hop_mmal_kernel<S, NC, false, EPI_SCHUR_TS, NTC, EXACT, PRE>; break;
        case EPI_SCHUR: k = hop_mmal_kernel<S, NC, false, EPI_SCHUR, NTC, EXACT, PRE>; break;
        case EPI_RESID: k = hop_mmal_kernel<S, NC, false, EPI_RESID, NTC, EXACT, PRE>; break;
        default: return set_error(QCU_ERR_INVALID, "epilogue %d", epi);
    }
    int grid = resident_grid(k, kLThreads, p.g.vh * nchunk * 32);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    k<<<grid, kLThreads, 0, st>>>(p, nchunk);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

// the staged kernel's blocks are 16-byte aligned in global memory
inline bool lalign16(const void* ptr) { return reinterpret_cast<uintptr_t>(ptr) % 16 == 0; }

template <typename S, int NC, int NTC>
int launch_mmal_f(const HopParams& p, bool dagger, int epi, int nchunk, bool staged, cudaStream_t st) {
    const bool pre = p.links != nullptr && p.nbr != nullptr;
    if (staged && pre && nchunk == 1 && p.m == 4 * NTC && lalign16(p.in) && lalign16(p.links) &&
        (!p.x || lalign16(p.x)) && (!p.r0 || lalign16(p.r0)))
    {
        return launch_mmal_tma<S, NC, NTC>(p, dagger, epi, st);
    }
    if (p.m == 4 * NTC * nchunk)
        return pre ? launch_mmal_t<S, NC, NTC, true, true>(p, dagger, epi, nchunk, st)
                   : launch_mmal_t<S, NC, NTC, true, false>(p, dagger, epi, nchunk, st);
    return pre ? launch_mmal_t<S, NC, NTC, false, true>(p, dagger, epi, nchunk, st)
               : launch_mmal_t<S, NC, NTC, false, false>(p, dagger, epi, nchunk, st);
}

template <typename S, int NC>
int launch_mmal_nc(const HopParams& p, bool dagger, int epi, bool staged, cudaStream_t st) {
    // groups of 4 RHS, at most 4 groups per work unit; chunks balanced
    const int groups = (p.m + 3) / 4;
    const int nchunk = (groups + 3) / 4;
    const int ntc = (groups + nchunk - 1) / nchunk;
    switch (ntc) {
        case 1: return launch_mmal_f<S, NC, 1>(p, dagger, epi, nchunk, staged, st);
        case 2: return launch_mmal_f<S, NC, 2>(p, dagger, epi, nchunk, staged, st);
        case 3: return launch_mmal_f<S, NC, 3>(p, dagger, epi, nchunk, staged, st);
        default: return launch_mmal_f<S, NC, 4>(p, dagger, epi, nchunk, staged, st);
    }
}

template <typename S>
int launch_mmal(const HopParams& p, int nc, bool dagger, int epi, bool staged, cudaStream_t st) {
    switch (nc) {
        case 2: return launch_mmal_nc<S, 2>(p, dagger, epi, staged, st);
        case 3: return launch_mmal_nc<S, 3>(p, dagger, epi, staged, st);
        default: return launch_mmal_nc<S, 4>(p, dagger, epi, staged, st);
    }
}

}  // namespace

namespace {
template <typename S, int NC, int NTC>
cudaError_t mmal_tma_optin() {
    const int need = kTBarBytes + kTWarps * kTStages * tstage_bytes(NC, 4 * NTC, 2);
    const void* ks[8] = {tma_kernel_ptr<S, NC, NTC, EPI_PLAIN, false>(), tma_kernel_ptr<S, NC, NTC, EPI_PLAIN, true>(),
                         tma_kernel_ptr<S, NC, NTC, EPI_XPAY, false>(), tma_kernel_ptr<S, NC, NTC, EPI_XPAY, true>(),
                         tma_kernel_ptr<S, NC, NTC, EPI_SCHUR_R0, false>(),
                         tma_kernel_ptr<S, NC, NTC, EPI_SCHUR_TS, false>(),
                         tma_kernel_ptr<S, NC, NTC, EPI_SCHUR, false>(), tma_kernel_ptr<S, NC, NTC, EPI_RESID, false>()};
    for (const void* k : ks) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, need);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
template <typename S, int NC>
cudaError_t mmal_tma_optin_nc() {
    cudaError_t e = mmal_tma_optin<S, NC, 1>();
    if (e == cudaSuccess) e = mmal_tma_optin<S, NC, 2>();
    if (e == cudaSuccess) e = mmal_tma_optin<S, NC, 3>();
    if (e == cudaSuccess) e = mmal_tma_optin<S, NC, 4>();
    return e;
}
}  // namespace

// One-time set-up of the staged kernel (shared-memory opt-in above 48 KB, the device error
// flag); call outside graph capture.
int hop_mmal_prepare() {
    static bool done = false;
    if (done) return QCU_SUCCESS;
    cudaError_t e = mmal_tma_optin_nc<__half, 2>();
    if (e == cudaSuccess) e = mmal_tma_optin_nc<__half, 3>();
    if (e == cudaSuccess) e = mmal_tma_optin_nc<__half, 4>();
    if (e == cudaSuccess) e = mmal_tma_optin_nc<__nv_bfloat16, 2>();
    if (e == cudaSuccess) e = mmal_tma_optin_nc<__nv_bfloat16, 3>();
    if (e == cudaSuccess) e = mmal_tma_optin_nc<__nv_bfloat16, 4>();
    if (e != cudaSuccess) return set_error(QCU_ERR_CUDA, "staged hop shared-memory opt-in: %s", cudaGetErrorString(e));
    if (!device_error_flag()) return set_error(QCU_ERR_CUDA, "device error flag unavailable");
    done = true;
    return QCU_SUCCESS;
}

bool hop_mmal_supported(int nc, int m, int prec) {
    return (prec == QCU_PRECISION_HALF || prec == QCU_PRECISION_BF16) && nc >= 2 && nc <= 8 && m >= 1 &&
           m <= kMaxRhs;
}

int hop_mmal_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, bool staged, cudaStream_t st) {
    if (!hop_mmal_supported(nc, p.m, prec))
        return set_error(QCU_ERR_UNSUPPORTED, "link-operand tensor-core hop: n_color=%d m_rhs=%d precision=%d", nc,
                         p.m, prec);
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    if ((epi != EPI_PLAIN && !p.x) || ((epi == EPI_SCHUR_R0 || epi == EPI_RESID) && !p.r0))
        return set_error(QCU_ERR_INVALID, "link-operand tensor-core hop: epilogue operand missing");
    // 32-bit word offsets: every spinor word index below 2^31
    if (p.g.vh * 4 * nc * (int64_t)p.m >= ((int64_t)1 << 31) || p.g.vh * 8 * nc * nc >= ((int64_t)1 << 31))
        return set_error(QCU_ERR_UNSUPPORTED, "link-operand tensor-core hop: field beyond 2^31 complex");
    if (nc >= 5) return hop_mmal_big_launch(p, nc, prec, dagger, epi, st);
    if (prec == QCU_PRECISION_HALF) return launch_mmal<__half>(p, nc, dagger, epi, staged, st);
    return launch_mmal<__nv_bfloat16>(p, nc, dagger, epi, staged, st);
}

}  // namespace qcub