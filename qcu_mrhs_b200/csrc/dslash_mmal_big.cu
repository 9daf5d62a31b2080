// dslash_mmal_big.cu -- the link-operand tensor-core hop for 5 <= N <= 8 (fragment scheme in
// dslash_mmal.cuh).
#include "dslash_mmal.cuh"

namespace qcub {

namespace {

// ---------------------------------------------------------------------------------
// 5 <= N <= 8.  The sum and the diff rows are two M tiles of 16 rows, each ordered (re/im,
// colour): lane (g, t) holds row g (real part) and row g + 8 (imaginary part) of colour g, so
// its D fragments hold whole complex outputs.  The forward and backward colours are two K
// steps (slots t and t + 4 of a step: colours t and t + 4).  Per direction and group of 4 RHS,
// two MMAs add the forward and backward hop into the sum tile (one for all directions:
// spins 0 and 1 from columns h0 and h1) and two into the diff tile of the direction's class
// (x/y or z/t as for N <= 4, spin 3 negated between the two directions of a class).  A work
// unit is (site, up to 8 RHS).
constexpr int kBMaxGroups = 2;

// the phase code C applied to a raw link word: i w = (-w.im, w.re)
template <int C>
__device__ __forceinline__ uint32_t wphase(uint32_t w) {
    if (C == 0) return w;
    if (C == 1) return w ^ 0x80008000u;
    if (C == 2) return swap_halves(w) ^ 0x00008000u;
    return swap_halves(w) ^ 0x80000000u;
}
// A fragments of one K step from the lane's link elements w0 = W[g][t], w4 = W[g][t + 4]
// (rows g: re, g + 8: im; slots t, t + 4): emb re row (w.re, -w.im), emb im row (w.im, w.re)
__device__ __forceinline__ void bemb(uint32_t (&A)[4], uint32_t w0, uint32_t w4) {
    A[0] = w0 ^ 0x80000000u;
    A[1] = swap_halves(w0);
    A[2] = w4 ^ 0x80000000u;
    A[3] = swap_halves(w4);
}

// One direction of the large-N kernel for all groups of the unit: fw / bw point at the
// forward / backward neighbour site (plus the chunk's first RHS and the lane's column RHS);
// o0 / o4 are the lane's word offsets of (half spinor h, colour t / t + 4), c0 / c4 those of
// the projection partner spin.
template <typename S, int MU, int SF, int NTC, bool EXACT>
__device__ __forceinline__ void mmalb_dir(float (&Sq)[NTC][4], float (&Q)[NTC][4], const uint32_t* __restrict__ fw,
                                          const uint32_t* __restrict__ bw, int o0, int o4, int c0, int c4,
                                          const uint32_t (&As0)[4], const uint32_t (&As1)[4],
                                          const uint32_t (&Ad0)[4], const uint32_t (&Ad1)[4], uint32_t lmf,
                                          uint32_t lmb, int rb0, int q, int m, uint32_t gmask) {
    using M = LMma<S>;
    constexpr int SB = -SF;
    uint32_t w[NTC][8];
#pragma unroll
    for (int n = 0; n < NTC; ++n) {
        if (!((gmask >> n) & 1u)) continue;   // warp-uniform: absent or inactive group
        int d = 4 * n;
        if (!EXACT) d += min(0, m - 1 - (rb0 + 4 * n + q));
        w[n][0] = __ldg(fw + o0 + d);
        w[n][1] = __ldg(fw + c0 + d);
        w[n][2] = __ldg(fw + o4 + d);
        w[n][3] = __ldg(fw + c4 + d);
        w[n][4] = __ldg(bw + o0 + d);
        w[n][5] = __ldg(bw + c0 + d);
        w[n][6] = __ldg(bw + o4 + d);
        w[n][7] = __ldg(bw + c4 + d);
    }
#pragma unroll
    for (int n = 0; n < NTC; ++n) {
        if (!((gmask >> n) & 1u)) continue;
        const uint32_t hf0 = lproject<S, MU, SF>(w[n][0], w[n][1], lmf);
        const uint32_t hf4 = lproject<S, MU, SF>(w[n][2], w[n][3], lmf);
        const uint32_t hb0 = lproject<S, MU, SB>(w[n][4], w[n][5], lmb);
        const uint32_t hb4 = lproject<S, MU, SB>(w[n][6], w[n][7], lmb);
        M::mma(Sq[n], As0, hf0, hf4, Sq[n][0], Sq[n][1], Sq[n][2], Sq[n][3]);
        M::mma(Sq[n], As1, hb0, hb4, Sq[n][0], Sq[n][1], Sq[n][2], Sq[n][3]);
        M::mma(Q[n], Ad0, hf0, hf4, Q[n][0], Q[n][1], Q[n][2], Q[n][3]);
        M::mma(Q[n], Ad1, hb0, hb4, Q[n][0], Q[n][1], Q[n][2], Q[n][3]);
    }
}

template <typename S, int NC, bool DAG, int EPI, bool PRE>
__global__ void __launch_bounds__(kLThreads, 2) hop_mmal_big_kernel(const HopParams p, int nchunk) {
    constexpr int NTC = kBMaxGroups;
    constexpr bool EXACT = false;   // the last group of a unit may be partial or empty
    using M = LMma<S>;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int NVR = NV > 0 ? NV : 1;
    constexpr int NY = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : 0;
    constexpr uint32_t N2 = NC * NC;
    constexpr int SF = DAG ? 1 : -1;
    static_assert(NC >= 5 && NC <= 8 && NTC <= kBMaxGroups, "large-N hop: 5 <= N <= 8, up to 8 RHS per unit");
    if (skip_launch(p.done, p.gate)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3, hh = g & 1, q = g >> 1;
    const int m = p.m;
    const uint32_t SW = 4u * NC * (uint32_t)m;
    const int gc = min(g, NC - 1), t0 = min(t, NC - 1), t4 = min(t + 4, NC - 1);
    const uint32_t ok0 = (g < NC && t < NC) ? 0xffffffffu : 0u;
    const uint32_t ok4 = (g < NC && t + 4 < NC) ? 0xffffffffu : 0u;
    const bool sok = g < NC;
    const int o0 = (hh * NC + t0) * m, o4 = (hh * NC + t4) * m;
    const int c01_0 = ((3 - hh) * NC + t0) * m, c01_4 = ((3 - hh) * NC + t4) * m;
    const int c23_0 = ((2 + hh) * NC + t0) * m, c23_4 = ((2 + hh) * NC + t4) * m;
    const int os = gc * m + t;                   // spin s of (colour g, RHS t) at os + s N m
    const int osn = NC * m;
    const uint32_t m1f = hh ? unit_pair<S>(SF, SF) : unit_pair<S>(-SF, -SF);
    const uint32_t m2f = hh ? unit_pair<S>(SF, -SF) : unit_pair<S>(-SF, SF);
    const uint32_t m1b = m1f ^ 0x80008000u, m2b = m2f ^ 0x80008000u;

    const uint32_t vh = (uint32_t)p.g.vh;
    const int parity = p.parity;
    const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
    uint32_t* __restrict__ out = static_cast<uint32_t*>(p.out);
    const uint32_t* __restrict__ xv = static_cast<const uint32_t*>(p.x);
    const uint32_t* __restrict__ yv = static_cast<const uint32_t*>(p.r0);
    const uint32_t gblk = vh * N2;
    const size_t gmu = 2 * (size_t)gblk;
    const uint32_t tflip = p.t_sign < 0 ? 0x80008000u : 0u;
    const uint32_t lxh = (uint32_t)p.g.lxh, Ly = (uint32_t)p.g.L[1], Lz = (uint32_t)p.g.L[2],
                   Lt = (uint32_t)p.g.L[3];
    const uint32_t sy = lxh, sz = lxh * Ly, st = sz * Lz;

    const int64_t gw = (int64_t)blockIdx.x * kLWarps + warp;
    const int64_t nw = (int64_t)gridDim.x * kLWarps;
    const int chunk = (int)(gw % nchunk);
    const uint32_t site_stride = (uint32_t)(nw / nchunk);
    const uint32_t site0 = gw < (int64_t)site_stride * nchunk ? (uint32_t)(gw / nchunk) : vh;
    const int rb0 = chunk * NTC * 4;
    const uint32_t gmask = active_groups<NTC>(p.active, rb0, m);
    const uint32_t* __restrict__ in = static_cast<const uint32_t*>(p.in) + rb0 + q;

    float2 red[NTC][NVR];
#pragma unroll
    for (int n = 0; n < NTC; ++n)
#pragma unroll
        for (int k = 0; k < NVR; ++k) red[n][k] = make_float2(0.f, 0.f);

    for (uint32_t site = site0; site < vh; site += site_stride) {
        uint32_t nb[8];
        uint32_t wf0[4], wf4[4], wb0[4], wb4[4];
        if constexpr (PRE) {
            const uint4* nt = reinterpret_cast<const uint4*>(p.nbr) + ((size_t)parity * vh + site) * 2;
            const uint4 na = __ldg(nt), nc4 = __ldg(nt + 1);
            nb[0] = na.x; nb[1] = na.y; nb[2] = na.z; nb[3] = na.w;
            nb[4] = nc4.x; nb[5] = nc4.y; nb[6] = nc4.z; nb[7] = nc4.w;
            const uint32_t* lk = static_cast<const uint32_t*>(p.links) + ((size_t)parity * vh + site) * 8 * N2 +
                                 (uint32_t)(gc * NC);
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                wf0[mu] = __ldg(lk + 2 * mu * N2 + t0);
                wf4[mu] = __ldg(lk + 2 * mu * N2 + t4);
                wb0[mu] = __ldg(lk + (2 * mu + 1) * N2 + t0);
                wb4[mu] = __ldg(lk + (2 * mu + 1) * N2 + t4);
            }
        } else {
            const SiteXYZT c = site_coords(p.g, site);
            const uint32_t xh = (uint32_t)c.xh;
            const int xodd = (parity ^ (c.y + c.z + c.t)) & 1;
            const uint32_t row = site - xh;
            nb[0] = row + (xodd ? (xh + 1 == lxh ? 0u : xh + 1) : xh);
            nb[1] = row + (xodd ? xh : (xh == 0 ? lxh - 1 : xh - 1));
            nb[2] = site + sy - ((uint32_t)c.y + 1 == Ly ? Ly * sy : 0u);
            nb[3] = site - sy + ((uint32_t)c.y == 0 ? Ly * sy : 0u);
            nb[4] = site + sz - ((uint32_t)c.z + 1 == Lz ? Lz * sz : 0u);
            nb[5] = site - sz + ((uint32_t)c.z == 0 ? Lz * sz : 0u);
            const bool wf_t = ((uint32_t)c.t + 1 == Lt), wb_t = (c.t == 0);
            nb[6] = site + st - (wf_t ? Lt * st : 0u);
            nb[7] = site - st + (wb_t ? Lt * st : 0u);
            const uint32_t* gf = gauge + (size_t)parity * gblk + (size_t)site * N2 + gc * NC;
            const uint32_t* gb = gauge + (size_t)(1 - parity) * gblk + gc;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                wf0[mu] = __ldg(gf + mu * gmu + t0);
                wf4[mu] = __ldg(gf + mu * gmu + t4);
                const uint32_t* ub = gb + mu * gmu + (size_t)nb[2 * mu + 1] * N2;
                wb0[mu] = __ldg(ub + t0 * NC) ^ 0x80000000u;   // W_b[g][t] = conj(U_b[t][g])
                wb4[mu] = __ldg(ub + t4 * NC) ^ 0x80000000u;
            }
            if (wf_t) { wf0[3] ^= tflip; wf4[3] ^= tflip; }
            if (wb_t) { wb0[3] ^= tflip; wb4[3] ^= tflip; }
        }
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            wf0[mu] &= ok0; wb0[mu] &= ok0;
            wf4[mu] &= ok4; wb4[mu] &= ok4;
        }
        const size_t sbase = (size_t)site * SW + rb0;

        uint32_t xw[NTC][4], yw[NTC][4];
        if constexpr (EPI != EPI_PLAIN) {
#pragma unroll
            for (int n = 0; n < NTC; ++n) {
#pragma unroll
                for (int e = 0; e < 4; ++e) xw[n][e] = yw[n][e] = 0u;
                if (!((gmask >> n) & 1u)) continue;
                if (sok && (EXACT || rb0 + 4 * n + t < m)) {
                    const size_t o = sbase + os + 4 * n;
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        xw[n][e] = __ldg(xv + o + e * osn);
                        if (NY) yw[n][e] = __ldg(yv + o + e * osn);
                    }
                }
            }
        }

        float Sq[NTC][4], Qxy[NTC][4], Qzt[NTC][4];
#pragma unroll
        for (int n = 0; n < NTC; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e) Sq[n][e] = Qxy[n][e] = Qzt[n][e] = 0.f;
        uint32_t As0[4], As1[4], Ad0[4], Ad1[4];
#define QCUB_BIG_DIR(MU, Q, FNB, BNB, C0, C4, LMF, LMB)                                                       \
        bemb(As0, wf0[MU], wf4[MU]);                                                                          \
        bemb(As1, wb0[MU], wb4[MU]);                                                                          \
        bemb(Ad0, wphase<LRecon<MU, SF>::C2>(wf0[MU]), wphase<LRecon<MU, SF>::C2>(wf4[MU]));                  \
        bemb(Ad1, wphase<LRecon<MU, SF>::C2 ^ 1>(wb0[MU]), wphase<LRecon<MU, SF>::C2 ^ 1>(wb4[MU]));          \
        mmalb_dir<S, MU, SF, NTC, EXACT>(Sq, Q, in + (size_t)(FNB) * SW, in + (size_t)(BNB) * SW, o0, o4, C0, C4, \
                                         As0, As1, Ad0, Ad1, LMF, LMB, rb0, q, m, gmask)
        // y, then spin 3 (diff column h0: registers 0 and 2) negated, then x; z, then spin 3
        // (column h1: registers 1 and 3) negated, then t
        QCUB_BIG_DIR(1, Qxy, nb[2], nb[3], c01_0, c01_4, m1f, m1b);
#pragma unroll
        for (int n = 0; n < NTC; ++n) {
            Qxy[n][0] = -Qxy[n][0];
            Qxy[n][2] = -Qxy[n][2];
        }
        QCUB_BIG_DIR(0, Qxy, nb[0], nb[1], c01_0, c01_4, 0u, 0u);
        QCUB_BIG_DIR(2, Qzt, nb[4], nb[5], c23_0, c23_4, m2f, m2b);
#pragma unroll
        for (int n = 0; n < NTC; ++n) {
            Qzt[n][1] = -Qzt[n][1];
            Qzt[n][3] = -Qzt[n][3];
        }
        QCUB_BIG_DIR(3, Qzt, nb[6], nb[7], c23_0, c23_4, 0u, 0u);
#undef QCUB_BIG_DIR

#pragma unroll
        for (int n = 0; n < NTC; ++n) {
            if (!((gmask >> n) & 1u)) continue;
            const bool rok = sok && (EXACT || rb0 + 4 * n + t < m);
            const size_t o = sbase + os + 4 * n;
            float2 ov[4];
            ov[0] = make_float2(Sq[n][0], Sq[n][2]);
            ov[1] = make_float2(Sq[n][1], Sq[n][3]);
            ov[2] = make_float2(Qxy[n][1] + Qzt[n][0], Qxy[n][3] + Qzt[n][2]);
            ov[3] = make_float2(Qxy[n][0] + Qzt[n][1], Qxy[n][2] + Qzt[n][3]);
            if (!rok) continue;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                if constexpr (EPI == EPI_PLAIN) {
                    out[o + e * osn] = M::pack(ov[e].x, ov[e].y);
                } else {
                    const float a = (float)p.a;
                    const float2 xx = M::unpack(xw[n][e]);
                    float2 res;
                    if (EPI == EPI_XPAY) {
                        res = make_float2(xx.x + a * ov[e].x, xx.y + a * ov[e].y);
                    } else if (EPI == EPI_RESID) {
                        const float2 yy = M::unpack(yw[n][e]);
                        res = make_float2(yy.x - xx.x + a * ov[e].x, yy.y - xx.y + a * ov[e].y);
                    } else {
                        res = make_float2(xx.x - a * ov[e].x, xx.y - a * ov[e].y);
                    }
                    const uint32_t rs = M::pack(res.x, res.y);
                    out[o + e * osn] = rs;
                    if constexpr (NV > 0) {
                        const float2 rr = M::unpack(rs);
                        if (EPI == EPI_RESID) {
                            red[n][0].x += rr.x * rr.x + rr.y * rr.y;
                        } else if (EPI == EPI_SCHUR_R0) {   // <r0, out> = sum conj(r0) out
                            const float2 qq = M::unpack(yw[n][e]);
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
            double2 sum = make_double2(0.0, 0.0);
            for (int w = 0; w < kLWarps; ++w) {
                if ((int)(((int64_t)blockIdx.x * kLWarps + w) % nchunk) != ch) continue;
                sum.x += wsum[w][k][loc].x;
                sum.y += wsum[w][k][loc].y;
            }
            bsum[idx] = sum;
        }
        __syncthreads();
        publish_and_finish<NV>(bsum, m, p.red);
    }
}

template <typename S, int NC, bool PRE>
int launch_mmal_big_t(const HopParams& p, bool dagger, int epi, int nchunk, cudaStream_t st) {
    void (*k)(const HopParams, int) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop_mmal_big_kernel<S, NC, true, EPI_PLAIN, PRE> : hop_mmal_big_kernel<S, NC, false, EPI_PLAIN, PRE>; break;
        case EPI_XPAY: k = dagger ? hop_mmal_big_kernel<S, NC, true, EPI_XPAY, PRE> : hop_mmal_big_kernel<S, NC, false, EPI_XPAY, PRE>; break;
        case EPI_SCHUR_R0: k = hop_mmal_big_kernel<S, NC, false, EPI_SCHUR_R0, PRE>; break;
        case EPI_SCHUR_TS: k = hop_mmal_big_kernel<S, NC, false, EPI_SCHUR_TS, PRE>; break;
        case EPI_SCHUR: k = hop_mmal_big_kernel<S, NC, false, EPI_SCHUR, PRE>; break;
        case EPI_RESID: k = hop_mmal_big_kernel<S, NC, false, EPI_RESID, PRE>; break;
        default: return set_error(QCU_ERR_INVALID, "epilogue %d", epi);
    }
    int grid = resident_grid(k, kLThreads, p.g.vh * nchunk * 32);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    k<<<grid, kLThreads, 0, st>>>(p, nchunk);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

// work units of up to 8 RHS (two groups of 4)
template <typename S, int NC>
int launch_mmal_big(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    const int nchunk = (p.m + 4 * kBMaxGroups - 1) / (4 * kBMaxGroups);
    const bool pre = p.links != nullptr && p.nbr != nullptr;
    return pre ? launch_mmal_big_t<S, NC, true>(p, dagger, epi, nchunk, st)
               : launch_mmal_big_t<S, NC, false>(p, dagger, epi, nchunk, st);
}

template <typename S>
int launch_mmal_big_nc(const HopParams& p, int nc, bool dagger, int epi, cudaStream_t st) {
    switch (nc) {
        case 5: return launch_mmal_big<S, 5>(p, dagger, epi, st);
        case 6: return launch_mmal_big<S, 6>(p, dagger, epi, st);
        case 7: return launch_mmal_big<S, 7>(p, dagger, epi, st);
        case 8: return launch_mmal_big<S, 8>(p, dagger, epi, st);
        default: return set_error(QCU_ERR_UNSUPPORTED, "large-N link-operand hop: n_color=%d", nc);
    }
}

}  // namespace

// operands, epilogue and size checks are done by hop_mmal_launch
int hop_mmal_big_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st) {
    if (prec == QCU_PRECISION_HALF) return launch_mmal_big_nc<__half>(p, nc, dagger, epi, st);
    return launch_mmal_big_nc<__nv_bfloat16>(p, nc, dagger, epi, st);
}

}  // namespace qcub
