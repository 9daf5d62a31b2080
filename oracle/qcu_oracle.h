/*
 * qcu_oracle.h -- CPU restatement of the multi-right-hand-side Wilson hop term,
 * the Wilson-Dirac operator, the even/odd Schur BiCGStab and the multi-RHS BLAS
 * of qcu_mrhs.
 *
 * THIS IS TEST INFRASTRUCTURE.  It is the correctness checker for the CUDA
 * library in qcu_mrhs_b200/ and the timed CPU baseline.  The product never links,
 * loads or calls it.
 *
 * Pinning: the reference ships no CPU dslash, no CPU solver and no golden
 * vectors for this path.  The conventions here are pinned (a) by analytic
 * known-answer tests (free-field plane wave, gauge covariance, gamma5
 * hermiticity, antiperiodic-link equivalence, M x = b), and (b) against the
 * reference's own CUDA hop kernels compiled from their sources with shim headers
 * (oracle/ref_build.sh) and run on a B200; the outputs are committed as
 * fixtures under tests/golden/.
 *
 * All complex arrays are interleaved (re, im) doubles.
 * Lattice dims L[4] = {Lx, Ly, Lz, Lt}; Lx even; Vh = Lx*Ly*Lz*Lt/2.
 *
 * Layouts (reference include/point/qcu_point.cuh:68-81,
 *          include/kernel/copy_vector/copy_color_spinor.cuh:27-37):
 *   half-site index  idx = ((t*Lz + z)*Ly + y)*(Lx/2) + xh
 *   full x           x   = 2*xh + ((parity + y + z + t) & 1)
 *   gauge            [mu=4][parity=2][Vh][Nc][Nc]           (row-major colour)
 *   per-RHS fermion  [parity=2][Vh][Ns=4][Nc]               (full lattice)
 *   gathered MRHS    [Vh][Ns=4][Nc][m]                      (one parity)
 */
#ifndef QCU_ORACLE_H
#define QCU_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Hop term D_p on the gathered layout (one output parity).
 * out(x) = sum_mu U_mu(x)(1 - s g_mu) in(x+mu) + U_mu(x-mu)^dag (1 + s g_mu) in(x-mu),
 * s = +1 (dagger = 0) or -1 (dagger = 1); hops that wrap in t get factor t_sign. */
void oracle_hop_mrhs(double* out, const double* in, const double* gauge, const int L[4],
                     int nc, int m, int parity, int dagger, double t_sign);

/* gather m per-RHS half-lattice fields [m][Vh][4][Nc] -> [Vh][4][Nc][m] and back */
void oracle_gather(double* mrhs, const double* per_rhs, long vh, int nc, int m);
void oracle_scatter(double* per_rhs, const double* mrhs, long vh, int nc, int m);

/* Full Wilson-Dirac operator M = 1 - kappa*D on m per-RHS EO full-lattice fields
 * laid out [m][2][Vh][4][Nc] (reference src/qcu_interface.cu:174-256). */
void oracle_mat(double* out, const double* in, const double* gauge, const int L[4],
                int nc, int m, double kappa, int dagger, double t_sign);

/* Schur operator A = 1 - kappa^2 D_oe D_eo on the odd gathered half lattice
 * (reference src/solver/bicgstab_solve.cu:27-70). tmp: one half-lattice MRHS vector. */
void oracle_schur(double* out, const double* in, double* tmp, const double* gauge,
                  const int L[4], int nc, int m, double kappa, double t_sign);

/* Multi-RHS BLAS on strided vectors: element i of RHS j at complex offset i*m + j.
 * len = number of complex elements per RHS. Scalars are complex arrays of length m. */
void oracle_dotc(double* res, const double* a, const double* b, long len, int m);
void oracle_norm(double* res, const double* a, long len, int m);
void oracle_xsay(double* res, const double* x, const double* a, const double* y, long len, int m);
void oracle_xpay(double* res, const double* x, const double* a, const double* y, long len, int m);
void oracle_axpby(double* res, const double* a, const double* x, const double* b,
                  const double* y, long len, int m);
void oracle_axpbypcz(double* res, const double* a, const double* x, const double* b,
                     const double* y, const double* c, const double* z, long len, int m);

/* Even/odd Schur BiCGStab, policy 1 (per-RHS scalars), x0 = 0, stop when every RHS
 * has recursive Schur residual ||r_j|| / ||b'_j|| <= tol
 * (reference src/solver/bicgstab_solve.cu:102-389, 688-740; bicgstab.cu:141-189).
 * b, x: gathered full lattice [2][Vh][4][Nc][m] (even half first).
 * Returns iterations used (>= 0) or -1 if max_iter was reached without convergence.
 * rel_resid (length m, may be NULL): final recursive ||r_j|| / ||b'_j||. */
int oracle_bicgstab(double* x, const double* b, const double* gauge, const int L[4], int nc,
                    int m, double kappa, double t_sign, int max_iter, double tol,
                    double* rel_resid);

/* Gauge reorder lexicographic [mu][t][z][y][x][Nc][Nc] <-> EO [mu][p][Vh][Nc][Nc]. */
void oracle_gauge_to_eo(double* eo, const double* lex, const int L[4], int nc);
void oracle_gauge_from_eo(double* lex, const double* eo, const int L[4], int nc);
/* Fermion reorder lexicographic [t][z][y][x][4][Nc] <-> EO [p][Vh][4][Nc]. */
void oracle_fermion_to_eo(double* eo, const double* lex, const int L[4], int nc);
void oracle_fermion_from_eo(double* lex, const double* eo, const int L[4], int nc);

/* Gauge-covariant parallel-transport convolution, the layer of the learned
 * preconditioner (no reference code; restated from its definition).
 * Fields: `ch` channels of gathered full-lattice multi-RHS spinors [ch][2][Vh][4][Nc][m].
 * Weights w[cout][cin][9][4][4] complex, one 4x4 spin matrix per (out, in, path).
 * Path k: 0 identity; 1 + 2 mu: U_mu(x) f(x + mu); 2 + 2 mu: U_mu(x - mu)^dag f(x - mu);
 * a hop that wraps in t is multiplied by t_sign.
 *   forward:  out_o(x) = sum_i sum_k w[o][i][k] (T_k in_i)(x)
 *   adjoint:  gin_i    = sum_o sum_k w[o][i][k]^dag T_k^dag gout_o   (T_k^dag = T_{-k})
 *   wgrad:    gw[o][i][k][s'][s] = sum_{x,c,r} gout_o(x)[s'][c][r] conj((T_k in_i)(x)[s][c][r])
 * For a real loss with gout = dLoss/d(out*), the gradient with respect to the real and
 * imaginary parts of w is 2 Re(gw), 2 Im(gw). */
void oracle_ptc_forward(double* out, const double* in, const double* w, const double* gauge,
                        const int L[4], int nc, int m, int cin, int cout, double t_sign);
void oracle_ptc_adjoint(double* gin, const double* gout, const double* w, const double* gauge,
                        const int L[4], int nc, int m, int cin, int cout, double t_sign);
void oracle_ptc_wgrad(double* gw, const double* gout, const double* in, const double* gauge,
                      const int L[4], int nc, int m, int cin, int cout, double t_sign);

/* Threads used by the OpenMP loops (0 = runtime default). */
void oracle_set_threads(int n);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
