// precond.h -- learned gauge-covariant preconditioner (internal host API).
//
// P is a stack of parallel-transport convolutions, channels 1 -> C -> ... -> C -> 1:
//   out_o(x) = sum_i sum_k W[o][i][k] (T_k in_i)(x),
//   T_0 = 1,  T_{1+2mu} f(x) = U_mu(x) f(x+mu),  T_{2+2mu} f(x) = U_mu(x-mu)^dag f(x-mu),
// W[o][i][k] a complex 4x4 spin matrix.  There is no nonlinearity, so P is a fixed linear
// operator that commutes with gauge transformations.  Fields are gathered full-lattice
// multi-RHS spinors [ch][2][Vh][4][Nc][m] (even half first) in FP32; weights are FP32
// complex, layer-major [layer][cout][cin][9][4][4].
#pragma once

#include <vector>

#include "context.h"

namespace qcub {

struct Precond {
    Geom g{};
    int nc = 3, m = 1, layers = 0, ch = 0;
    double t_sign = 1.0;
    std::vector<int> cin, cout;
    std::vector<int64_t> woff;      // complex offset of each layer's weights
    int64_t nw = 0;                 // complex weights in total
    DevBuf w, wadj, gw, m1, m2;     // weights, adjoint weights, gradient (double2), Adam moments
    DevBuf gauge;                   // FP32 gauge of the training API
    bool has_gauge = false;
    DevBuf act;                     // layer inputs/outputs: 1 + C (layers - 1) + 1 fields
    DevBuf gbuf[2];                 // gradient ping-pong, C fields each
    DevBuf tmp[3];                  // loss temporaries (one field each)
    DevBuf norms;                   // device double[2 * kMaxRhs]
    double* host_norms = nullptr;   // pinned mirror
    Scratch ws;
    cudaStream_t stream = nullptr;
    int step = 0;

    int64_t field_len() const { return 2 * g.vh * 4 * nc * (int64_t)m; }   // complex per channel
    size_t field_bytes() const { return (size_t)field_len() * sizeof(float2); }
    int act_offset(int l) const { return l == 0 ? 0 : 1 + (l - 1) * ch; }  // field index of layer l input

    int init(const int L[4], int n_color, int m_rhs, int n_layers, int channels, double t_boundary);
    void release();
    // out = P in (FP32 fields); gauge: FP32 EO gauge; kernels return at once once *done is set
    int apply(float2* out, const float2* in, const void* gauge32, cudaStream_t st, const int* done = nullptr);
    // loss = sum_j ||M P b_j - b_j||^2 / ||b_j||^2 and the weight gradient into gw
    int loss_grad(const float2* b, double kappa, double* loss, cudaStream_t st);
    int adam(double lr, cudaStream_t st);
};

// Right-preconditioned BiCGStab on the full system M x = b (solver.cu).
int solve_precond(Context& c, Precond* P, void* x, const void* b, int max_iter, double tol);

// ---- FP64 BiCGStab pieces of the preconditioned solve (precond.cu) ----
// alpha = rho / <r0, v>
int pc_alpha(const void* r0, const void* v, BicgScalars* sc, int64_t len, int m, const Scratch& ws, cudaStream_t st);
// omega = <t, s> / <t, t>
int pc_omega(const void* t, const void* s, BicgScalars* sc, int64_t len, int m, const Scratch& ws, cudaStream_t st);
// x += alpha ph + omega sh ; r = s - omega t ; |r|^2, <r0, r>, beta, convergence
int pc_xr(void* x, void* r, const void* ph, const void* sh, const void* s, const void* t, const void* r0,
          BicgScalars* sc, int64_t len, int m, const Scratch& ws, cudaStream_t st);
// FP64 <-> FP32 copy that returns at once once *done is set
int pc_cast(void* dst, int dprec, const void* src, int sprec, int64_t n, const int* done, cudaStream_t st);
// full-lattice M = 1 - kappa D (or M^dag) on gathered fields in `prec`
int full_mat(void* out, const void* in, const void* gauge, const Geom& g, int nc, int m, double kappa,
             double t_sign, bool dagger, int prec, cudaStream_t st, const int* done = nullptr);

}  // namespace qcub
