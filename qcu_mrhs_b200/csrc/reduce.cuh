// reduce.cuh -- deterministic per-RHS grid reductions with a last-block finisher,
// and the device-resident BiCGStab scalars that the finishers update.
//
// Every reducing kernel here uses a block size that is a multiple of m and a
// grid-stride loop whose stride is a multiple of m, so thread `tid` always works on
// RHS `tid % m`.  Each block writes its per-RHS partial sums to a scratch array;
// the last block to finish (atomic ticket) sums the partials in a fixed order,
// so results do not depend on block scheduling.
#pragma once

#include "common.cuh"

namespace qcub {

constexpr int kRedThreads = 256;    // max block size of reducing kernels
constexpr int kMaxRedVals = 3;      // values reduced per RHS by one kernel

// Device-resident state of the multi-RHS BiCGStab (reference scalars rho, alpha,
// omega, beta of src/solver/bicgstab_solve.cu:102-389, one per RHS).
struct BicgScalars {
    double2 rho[kMaxRhs];
    double2 alpha[kMaxRhs];
    double2 omega[kMaxRhs];
    double2 beta[kMaxRhs];
    double2 red[kMaxRedVals][kMaxRhs];  // raw output of the last reduction
    double bnorm2[kMaxRhs];             // ||b'_j||^2 (or the stopping reference)
    double rnorm2[kMaxRhs];             // ||r_j||^2 of the recursive residual
    double tol2;                        // stop when rnorm2 <= tol2 * bnorm2
    int active[kMaxRhs];                // 1 while RHS j still iterates
    int m;
    int freeze;                         // converged RHS stop updating
    int iter;                           // completed iterations
    int max_iter;
    int done;                           // kernels return immediately once set
    int status;                         // 0 running, 1 converged, 2 breakdown, 3 max_iter
    // ---- mixed precision (sloppy inner iteration, FP64 reliable updates) ----
    int mixed;                          // 1: FIN_BETA schedules reliable updates instead of stopping
    int gate;                           // 1: a reliable update is pending
    int reliable;                       // reliable updates done
    int restart;                        // 1: the pending update also resets p and r0 (breakdown)
    int x_fresh;                        // 1: the next STEP_XR writes the FP32 increment instead of
                                        //    adding to it (it was just folded into the FP64 x)
    double delta;                       // update when ||r_j|| < delta * maxr_j
    double quorum;                      // fraction of the active RHS that must meet the delta
                                        // rule (0: any one RHS)
    double len_per_rhs;                 // complex elements per RHS of the sloppy vectors
    double scale[kMaxRhs];              // sloppy vectors hold scale_j * (FP64 quantity)
    double ratio[kMaxRhs];              // scale_new / scale_old of the last update
    double maxr[kMaxRhs];               // max sloppy ||r_j|| since the last update
    double bfull2[kMaxRhs];             // ||b_j||^2 of the full system (stopping reference)
    double rtrue2[kMaxRhs];             // ||b' - A x||^2 at the last reliable update
    double beta_max;                    // |beta| above it counts as a sloppy breakdown
    double best2[kMaxRhs];              // smallest rtrue2 so far (stagnation guard)
    int stall[kMaxRhs];                 // reliable updates since rtrue2 last fell below 0.98 best2
};

// Mixed solver guards.  With FP16 storage a sloppy |beta| above kMaxHalfBeta (omega near
// zero) counts as a breakdown: p = r + beta (p - omega v) would leave the FP16 range, so
// the pending reliable update restarts p and r0 from the FP64 residual instead (BF16 and
// FP32 share the FP32 exponent range and take no such bound).  The solve stops as not
// converged (status 4) once an unconverged RHS's FP64 residual has not fallen by 2% over
// kStallUpdates reliable updates in a row.
constexpr double kMaxHalfBeta = 1e3;
constexpr int kStallUpdates = 32;

enum Finisher : int {
    FIN_NONE = 0,     // only publish the sums into sc->red (or the result array)
    FIN_ALPHA = 1,    // alpha_j = rho_j / <r0, v>_j
    FIN_OMEGA = 2,    // omega_j = <t, s>_j / <t, t>_j
    FIN_BETA = 3,     // rnorm2, convergence, beta_j = (alpha_j rho'_j / omega_j) / rho_j, rho <- rho'
    FIN_INIT = 4,     // rho_j = <r0, r0>_j = ||b'_j||^2 ; bnorm2 from the norm
    FIN_NORM = 5,     // norm_out[j] = sqrt(sum_j)
    FIN_RNORM = 6,    // sc->rtrue2[j] = sum_j (true residual of the reliable update)
    FIN_RHO = 7,      // sc->rho[j] = sum_j ; sc->gate = 0 (reliable update finished)
};

struct RedArgs {
    double2* partials;   // [gridDim][nval][m] scratch
    unsigned* counter;   // zero before the launch; reset to zero by the last block
    double2* result;     // [nval][m] output (may alias sc->red)
    BicgScalars* sc;     // for finishers (may be null with FIN_NONE / FIN_NORM)
    double* norm_out;    // FIN_NORM output [m]
    int fin;
};

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ bool cfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// Solver scalar updates, run by the last block after the sums are final.
__device__ inline void run_finisher(const RedArgs& ra, int m, const double2* sums) {
    BicgScalars* sc = ra.sc;
    const int tid = threadIdx.x;
    if (ra.fin == FIN_NORM) {
        if (tid < m) ra.norm_out[tid] = sqrt(sums[tid].x);
        return;
    }
    if (ra.fin == FIN_RNORM) {
        if (tid < m) sc->rtrue2[tid] = sums[tid].x;
        return;
    }
    if (ra.fin == FIN_RHO) {
        if (tid < m) sc->rho[tid] = sums[tid];
        __syncthreads();
        if (tid == 0) {
            sc->gate = 0;
            sc->restart = 0;
        }
        return;
    }
    __shared__ int s_flags[2];
    __shared__ int s_cnt[2];   // mixed: RHS that met the reliable-update rule, active RHS
    if (tid == 0) { s_flags[0] = 1; s_flags[1] = 0; s_cnt[0] = 0; s_cnt[1] = 0; }   // all converged, breakdown
    __syncthreads();
    if (tid < m) {
        const int j = tid;
        const bool act = sc->active[j] != 0;
        switch (ra.fin) {
            case FIN_INIT: {
                sc->bnorm2[j] = sums[j].x;
                sc->rho[j] = make_double2(sums[j].x, 0.0);
                sc->rnorm2[j] = sums[j].x;
                if (!(sums[j].x > 0.0)) sc->active[j] = 0;  // zero source: x_j = 0
            } break;
            case FIN_ALPHA: {
                double2 a = act ? cdiv(sc->rho[j], sums[j]) : make_double2(0.0, 0.0);
                if (act && !cfinite(a)) { s_flags[1] = 1; a = make_double2(0.0, 0.0); }
                sc->alpha[j] = a;
            } break;
            case FIN_OMEGA: {
                double2 w = act ? cdiv(sums[j], sums[m + j]) : make_double2(0.0, 0.0);
                if (act && !cfinite(w)) { s_flags[1] = 1; w = make_double2(0.0, 0.0); }
                sc->omega[j] = w;
            } break;
            case FIN_BETA: {
                const double rn2 = sums[j].x;
                const double2 rho_new = sums[m + j];
                if (sc->mixed) {
                    // sloppy recursive residual: schedule a reliable update when it fell by
                    // delta since the last one, or when it claims convergence (checked in FP64)
                    double2 b = make_double2(0.0, 0.0);
                    if (act) {
                        sc->rnorm2[j] = rn2;
                        const double rn = sqrt(rn2);
                        if (rn > sc->maxr[j]) sc->maxr[j] = rn;
                        const double sj = sc->scale[j];
                        atomicAdd(&s_cnt[1], 1);
                        if (rn < sc->delta * sc->maxr[j] || rn2 <= sc->tol2 * sc->bfull2[j] * sj * sj)
                            atomicAdd(&s_cnt[0], 1);
                        // far past the threshold: update whatever the quorum
                        if (rn < sc->delta * sc->delta * sc->maxr[j])
                            s_flags[0] = 0;   // reused below as "update forced" (inverted)
                        b = cdiv(cmul(sc->alpha[j], rho_new), sc->omega[j]);
                        b = cdiv(b, sc->rho[j]);
                        if (!cfinite(b) || !(b.x * b.x + b.y * b.y <= sc->beta_max * sc->beta_max) ||
                            !isfinite(rn2)) {
                            s_flags[1] = 1;
                            b = make_double2(0.0, 0.0);
                        }
                        sc->rho[j] = rho_new;
                    }
                    sc->beta[j] = b;
                    break;
                }
                if (act) sc->rnorm2[j] = rn2;
                // frozen RHS keep the norm they converged with, so `conv` stays true;
                // without freezing every RHS keeps iterating until all converge at once
                // (reference isConverged, bicgstab_solve.cu:77-88)
                const bool conv = sc->rnorm2[j] <= sc->tol2 * sc->bnorm2[j];
                if (!conv) atomicAnd(&s_flags[0], 0);
                double2 b = make_double2(0.0, 0.0);
                if (act) {
                    b = cdiv(cmul(sc->alpha[j], rho_new), sc->omega[j]);
                    b = cdiv(b, sc->rho[j]);
                    if (!cfinite(b) && !conv) s_flags[1] = 1;
                    if (!cfinite(b)) b = make_double2(0.0, 0.0);
                    sc->rho[j] = rho_new;
                    if (conv && sc->freeze) sc->active[j] = 0;
                }
                sc->beta[j] = b;
            } break;
            default: break;
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (ra.fin == FIN_BETA && sc->mixed) {
            sc->iter += 1;
            // enough RHS met the rule (any one with quorum 0), one is far past it, or a
            // breakdown: schedule a reliable update
            int need = 1;
            if (sc->quorum > 0.0) {
                need = (int)ceil(sc->quorum * (double)s_cnt[1] - 1e-9);
                if (need < 1) need = 1;
            }
            if (s_cnt[0] >= need || !s_flags[0] || s_flags[1]) sc->gate = 1;
            if (s_flags[1]) sc->restart = 1;
            if (sc->iter >= sc->max_iter) { sc->status = 3; sc->done = 1; }
        } else if (ra.fin == FIN_BETA) {
            sc->iter += 1;
            if (s_flags[0]) { sc->status = 1; sc->done = 1; }
            else if (s_flags[1]) { sc->status = 2; sc->done = 1; }
            else if (sc->iter >= sc->max_iter) { sc->status = 3; sc->done = 1; }
        } else if ((ra.fin == FIN_ALPHA || ra.fin == FIN_OMEGA) && s_flags[1]) {
            if (sc->mixed) {          // sloppy breakdown: recompute in FP64 and restart
                sc->gate = 1;
                sc->restart = 1;
            } else {
                sc->status = 2;
                sc->done = 1;
            }
        }
    }
}

// Grid stage of a reduction: every block publishes its per-RHS sums `bsum` (shared
// memory, [NV][m], final for this block), the last block to arrive sums all blocks'
// partials in a fixed order, writes the result and runs the finisher.
// Must be called by every thread of the block, exactly once per launch.
template <int NV>
__device__ inline void publish_and_finish(const double2* bsum, int m, const RedArgs& ra) {
    __shared__ bool s_last;
    const int tid = threadIdx.x;
    const int nb = blockDim.x;
    for (int idx = tid; idx < NV * m; idx += nb) ra.partials[(size_t)blockIdx.x * NV * m + idx] = bsum[idx];
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const unsigned ticket = atomicAdd(ra.counter, 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // last block: one warp per output value, lanes stride over blocks, fixed order
    // (only full warps take part: block sizes that are multiples of m may end in a
    // partial warp, which must not enter the full-mask shuffles)
    const int warp = tid >> 5, lane = tid & 31, nwarps = nb >> 5;
    __shared__ double2 fin[NV * kMaxRhs];
    for (int idx = warp; warp < nwarps && idx < NV * m; idx += nwarps) {
        double2 s = make_double2(0.0, 0.0);
        for (int b = lane; b < (int)gridDim.x; b += 32) {
            const double2 p = __ldcg(&ra.partials[(size_t)b * NV * m + idx]);
            s.x += p.x;
            s.y += p.y;
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            s.x += __shfl_down_sync(0xffffffffu, s.x, off);
            s.y += __shfl_down_sync(0xffffffffu, s.y, off);
        }
        if (lane == 0) fin[idx] = s;
    }
    __syncthreads();
    for (int idx = tid; idx < NV * m; idx += nb) ra.result[idx] = fin[idx];
    if (tid == 0) *ra.counter = 0u;
    __syncthreads();
    if (ra.fin != FIN_NONE) run_finisher(ra, m, fin);
}

// Block + grid reduction of NV double2 values per thread.  Thread tid works on RHS
// (tid / g) % m (g = 1: tid % m; the colour-split hop has g = n_color).
// Must be called by every thread of the block, exactly once per launch.
template <int NV>
__device__ inline void grid_reduce(const double2 (&v)[NV], int m, const RedArgs& ra, int g = 1) {
    __shared__ double2 sh[NV * kRedThreads];
    __shared__ double2 bsum[NV * kMaxRhs];
    const int tid = threadIdx.x;
    const int nb = blockDim.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k * nb + tid] = v[k];
    __syncthreads();
    for (int idx = tid; idx < NV * m; idx += nb) {
        const int k = idx / m, j = idx - (idx / m) * m;
        double2 s = make_double2(0.0, 0.0);
        for (int base = j * g; base < nb; base += g * m)
            for (int l = 0; l < g && base + l < nb; ++l) {
                s.x += sh[k * nb + base + l].x;
                s.y += sh[k * nb + base + l].y;
            }
        bsum[idx] = s;
    }
    __syncthreads();
    publish_and_finish<NV>(bsum, m, ra);
}

// Block size for a kernel whose thread works on RHS tid % m: largest multiple of m <= cap.
inline int rhs_block(int m, int cap = kRedThreads) { return (cap / m) * m; }

}  // namespace qcub
