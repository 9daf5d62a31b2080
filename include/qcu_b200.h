/*
 * qcu_b200.h -- extensions of the qcu.h interface in libqcu_b200.so.
 *
 * Three groups:
 *   1. status reporting, solver options and solve statistics for the qcu.h entry
 *      points (the reference reports errors by aborting and has no options);
 *   2. device-level entry points on caller-owned device buffers, one per reference
 *      operator on the hot path (each cites the reference interface it replaces);
 *   3. precision codes.
 * All functions return a status code (QCU_SUCCESS = 0) unless stated otherwise.
 * `stream` arguments are cudaStream_t values passed as void* (NULL = legacy stream).
 */
#pragma once

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- precision codes (reference enum QcuPrecision: half, single, double, undefined;
 *      its numeric values live in a header outside the reference tree) ---- */
#define QCU_PRECISION_HALF 0
#define QCU_PRECISION_SINGLE 1
#define QCU_PRECISION_DOUBLE 2
#define QCU_PRECISION_UNDEFINED 3
#define QCU_PRECISION_BF16 4 /* extension: bfloat16 storage, fp32 arithmetic */

/* reference qcu_helper_macro.h:7-11 */
#define QCU_DSLASH_WILSON 0

/* ---- status codes ---- */
#define QCU_SUCCESS 0
#define QCU_ERR_INVALID 1        /* bad argument (size, precision, pointer) */
#define QCU_ERR_STATE 2          /* wrong call order (not initialised, queue not full, ...) */
#define QCU_ERR_CUDA 3           /* CUDA runtime error */
#define QCU_ERR_NOT_CONVERGED 4  /* solver hit max_iteration */
#define QCU_ERR_BREAKDOWN 5      /* solver breakdown (rho, omega or <r0,v> vanished / not finite) */
#define QCU_ERR_UNSUPPORTED 6    /* feature not available */
#define QCU_ERR_ALLOC 7          /* device allocation failed */

/* Status of the most recent qcu.h / qcu_b200.h call on this process. */
int qcuGetLastStatus(void);
/* Human-readable message for the most recent failure ("" after success). */
const char *qcuGetLastError(void);

/* ---- solver selection for qcuInvert ---- */
#define QCU_SOLVER_REFERENCE 0 /* reference policy-1 BiCGStab, output precision, recursive residual */
#define QCU_SOLVER_FUSED 1     /* same iteration, fused device-resident kernels, CUDA graph */
#define QCU_SOLVER_MIXED 2     /* sloppy-precision inner BiCGStab with FP64 reliable updates; a
                                  sloppy breakdown restarts from the FP64 residual, and an FP64
                                  residual that stops falling (no 2% gain over 32 reliable
                                  updates) ends the solve with QCU_ERR_NOT_CONVERGED */
#define QCU_SOLVER_PRECOND 3   /* FP64 BiCGStab on the full system, right-preconditioned by the
                                  learned preconditioner of qcuSetPreconditioner; falls back to
                                  QCU_SOLVER_FUSED if it does not converge */
#define QCU_SOLVER_CGNR 4      /* conjugate gradients on the normal equations of the Schur
                                  system, A^dag A x = A^dag b' (A^dag from the dagger hops) */

typedef struct {
    int solver;              /* QCU_SOLVER_* (default QCU_SOLVER_FUSED) */
    int sloppy_precision;    /* inner precision for QCU_SOLVER_MIXED (QCU_PRECISION_*) */
    int stop_true_residual;  /* 1: stop on FP64 true residual ||b - M x|| / ||b|| (full system);
                                0: reference rule, recursive Schur residual ||r_o|| / ||b'_o|| */
    double reliable_delta;   /* MIXED: reliable update when ||r|| < delta * max ||r|| (0.1) */
    double t_boundary;       /* +1 periodic in t (reference), -1 antiperiodic in t */
    int check_interval;      /* iterations per captured graph between host checks (8) */
    int freeze_converged;    /* 1: converged right-hand sides stop updating (the MIXED solver
                                always stops an RHS whose FP64 residual converged, and its
                                tensor-core sloppy hops skip groups of 4 stopped RHS) */
    int max_restarts;        /* MIXED: cap on reliable updates (0 = unlimited) */
    double reliable_quorum;  /* MIXED: a reliable update waits until this fraction of the
                                unconverged RHS met the delta rule or claim convergence
                                (0: any one RHS, the default); an RHS whose sloppy residual
                                fell below delta^2 * max ||r|| forces the update */
} QcuSolverOptions;

void qcuGetDefaultSolverOptions(QcuSolverOptions *opts);
/* Applies to the next qcuInvert / mat_Qcu / start_dslash of the current context. */
int qcuSetSolverOptions(const QcuSolverOptions *opts);

#define QCU_MAX_RHS 64

typedef struct {
    int iterations;          /* BiCGStab iterations (sloppy iterations for MIXED) */
    int reliable_updates;    /* MIXED only */
    int status;              /* QCU_SUCCESS, QCU_ERR_NOT_CONVERGED or QCU_ERR_BREAKDOWN */
    int m_rhs;
    double true_residual[QCU_MAX_RHS];      /* ||b - M x|| / ||b|| per RHS, full system, FP64 */
    double recursive_residual[QCU_MAX_RHS]; /* last recursive Schur residual ||r|| / ||b'|| */
    double solve_seconds;    /* device time of the solve (gather..scatter), CUDA events */
    int fallback;            /* PRECOND: 1 when the plain solver had to finish the solve */
    int precond_iterations;  /* PRECOND: iterations of the preconditioned BiCGStab */
} QcuSolveStats;

/* Statistics of the last qcuInvert on the current context. */
int qcuGetSolveStats(QcuSolveStats *stats);

/* ---- batched solves of independent systems ----
 * No counterpart in the reference (its Qcu object holds one system).  Each system has
 * its own lattice, colour count, RHS count, kappa, tolerance and gauge field; all are
 * solved together on the current GPU with the even/odd Schur BiCGStab selected by
 * `opts` (NULL: defaults), one CUDA graph holding every system as an independent
 * branch.  Fields are FP64 device pointers in the qcu.h layouts: gauge EO
 * [4][2][Vh][N][N], each b[j] / x[j] a full-lattice EO fermion [2][Vh][4][N].
 * Outputs are written into the struct.  Returns QCU_SUCCESS when every system
 * converged, else the first failing status (every x is still written). */
typedef struct {
    int lattice_size[4];    /* X, Y, Z, T */
    int n_color;
    int m_rhs;
    double kappa;
    double tol;             /* per-RHS relative tolerance, as in qcuInvert */
    int max_iteration;
    const void *gauge;
    void *const *b;         /* m_rhs source pointers */
    void *const *x;         /* m_rhs solution pointers */
    /* outputs */
    int iterations;
    int reliable_updates;
    int status;
    double true_residual_max;  /* max_j ||b_j - M x_j|| / ||b_j|| (FP64) */
    double latency_seconds;    /* from the start of the iterations to this system's convergence */
} QcuBatchSystem;

/* ---- learned gauge-covariant preconditioner ----
 * No counterpart in the reference.  P is a stack of `layers` parallel-transport
 * convolutions with channels 1 -> C -> ... -> C -> 1 and no nonlinearity, so it is a
 * fixed linear operator that commutes with gauge transformations:
 *   out_o(x) = sum_i sum_k W[o][i][k] (T_k in_i)(x),  k = 0..8,
 *   T_0 = 1,  T_{1+2mu} f(x) = U_mu(x) f(x+mu),  T_{2+2mu} f(x) = U_mu(x-mu)^dag f(x-mu)
 * (hops across the t boundary carry t_boundary), W[o][i][k] a complex 4x4 spin matrix.
 * Weights are FP32 complex (re, im interleaved), layer-major [layer][cout][cin][9][4][4].
 * Fields are gathered full-lattice multi-RHS spinors [2][Vh][4][N][m] (even half first)
 * on the device, FP32 or FP64.  Training minimises sum_j ||M P b_j - b_j||^2 / ||b_j||^2
 * (M = 1 - kappa D) with the library's own forward, adjoint and weight-gradient kernels
 * and Adam.  2 <= n_color <= 4. */
int qcuPrecondCreate(void **handle, const int L[4], int n_color, int m_rhs, int layers, int channels,
                     double t_boundary);
int qcuPrecondDestroy(void *handle);
/* number of complex weights (negative status on error) */
int64_t qcuPrecondNumWeights(void *handle);
/* host arrays of 2 * qcuPrecondNumWeights floats; setting the weights resets Adam */
int qcuPrecondSetWeights(void *handle, const float *weights);
int qcuPrecondGetWeights(void *handle, float *weights);
/* EO gauge field [4][2][Vh][N][N] on the device, kept as an FP32 copy */
int qcuPrecondSetGauge(void *handle, const void *gauge, int precision);
/* out = P in on `stream` */
int qcuPrecondApply(void *handle, void *out, const void *in, int precision, void *stream);
/* loss and, if grad is not NULL, d loss / d(Re w, Im w) as 2 * NumWeights doubles */
int qcuPrecondLossGrad(void *handle, const void *b, int precision, double kappa, double *loss, double *grad);
/* one Adam step (beta 0.9, 0.999) on the loss of the m right-hand sides b */
int qcuPrecondTrainStep(void *handle, const void *b, int precision, double kappa, double lr, double *loss);
/* attach P to the qcu.h context for QCU_SOLVER_PRECOND (NULL detaches); its lattice,
 * n_color and m_rhs must match the context's */
int qcuSetPreconditioner(void *handle);

/* flags of qcuInvertBatch */
#define QCU_BATCH_DEVICE_LOOP 0 /* one graph launch; each system loops in a conditional graph node */
#define QCU_BATCH_HOST_LOOP 1   /* the host relaunches the graph every check_interval iterations */
#define QCU_BATCH_KEEP_CONTEXTS 2 /* keep each system's context and device buffers after the call;
                                     a later batch reuses them for systems of the same lattice,
                                     n_color and m_rhs (qcuBatchRelease frees them) */

/* opts = NULL: the defaults of qcuGetDefaultSolverOptions with freeze_converged = 1 */
int qcuInvertBatch(QcuBatchSystem *systems, int n_systems, const QcuSolverOptions *opts, int flags);
/* free the contexts kept by QCU_BATCH_KEEP_CONTEXTS */
int qcuBatchRelease(void);

/* ---- device-level entry points (caller-owned device buffers) ----
 * Gathered multi-RHS layout, one parity: [Vh][4][Nc][m] complex.
 * Gauge: [4][2][Vh][Nc][Nc] complex in the same precision as the spinors.
 * L = {Lx, Ly, Lz, Lt}.  2 <= n_color <= 8, 1 <= m_rhs <= 64.
 */

/* Hop term out[parity] = D in[1 - parity] on gathered fields.
 * Replaces qcu::Dslash::apply -- reference include/qcd/qcu_dslash.h:56-74,
 * src/qcd/qcu_dslash_wilson.cu:36-59 (wmma) and src/qcd/qcu_wilson_dslash_simt.cu:68-89 (SIMT). */
int qcuDslashMrhs(void *out, const void *in, const void *gauge, const int L[4], int n_color,
                  int m_rhs, int parity, int dagger, double t_sign, int precision, void *stream);

/* out = x + a * D in  (the hop with the xpay epilogue of src/solver/bicgstab.cu:141-189). */
int qcuDslashMrhsXpay(void *out, const void *in, const void *gauge, const void *x, double a,
                      const int L[4], int n_color, int m_rhs, int parity, int dagger, double t_sign,
                      int precision, void *stream);

/* qcuDslashMrhs on the gauge field of the qcu.h context (initGridSize, loadQcuGauge,
 * getDslash), its lattice, n_color, m_rhs and t boundary (qcuSetSolverOptions), in
 * `precision`: the hop the context's solver runs, including, for the FP16/BF16 tensor-core
 * kernel, its per-site neighbour table and hop-link array (built on first use).  For
 * callers that keep their own gathered multi-RHS fields.  Counterpart of calling the
 * reference's qcu::Dslash::apply on the Qcu object's gauge copies
 * (src/qcu_interface.cu:109-172 without the gather/scatter). */
int qcuDslashMrhsContext(void *out, const void *in, int parity, int dagger, int precision, void *stream);
/* The same with per-RHS activity flags `active` (device int[m_rhs]): the FP16/BF16
 * tensor-core hop (QCU_HOP_MMA_LINK) skips every group of 4 RHS (0-3, 4-7, ...) whose flags
 * are all 0 and leaves their outputs as they were; other kernels compute every RHS.  The
 * mixed solver's sloppy hops run this way with the flags of its converged RHS. */
int qcuDslashMrhsContextActive(void *out, const void *in, int parity, int dagger, int precision,
                               const int *active, void *stream);
/* The context's hop with one of the fused epilogues its solvers run (the same kernels):
 *   PLAIN     out = D in
 *   XPAY      out = x + a D in
 *   SCHUR_R0  out = x - a D in, and red[j] = <r0_j, out_j>            (BiCGStab v = A p)
 *   SCHUR_TS  out = x - a D in, and red[j] = <out_j, x_j>, red[m + j] = <out_j, out_j>
 *   SCHUR     out = x - a D in
 *   RESID     out = r0 - (x - a D in), and red[j] = ||out_j||^2
 * red: device double2 array of (number of sums) x m_rhs, or NULL to discard the sums. */
#define QCU_HOP_FORM_PLAIN 0
#define QCU_HOP_FORM_XPAY 1
#define QCU_HOP_FORM_SCHUR_R0 2
#define QCU_HOP_FORM_SCHUR_TS 3
#define QCU_HOP_FORM_SCHUR 4
#define QCU_HOP_FORM_RESID 5
int qcuDslashMrhsContextForm(void *out, const void *in, const void *x, const void *r0, double a, int form,
                             int parity, int precision, void *red, void *stream);

/* Schur operator out_o = in_o - kappa^2 D_oe D_eo in_o; tmp is one half-lattice vector.
 * Replaces fused_x_sub_Doe_Deo_x -- reference src/solver/bicgstab_solve.cu:27-70. */
int qcuSchurMrhs(void *out, const void *in, void *tmp, const void *gauge, double kappa,
                 const int L[4], int n_color, int m_rhs, double t_sign, int precision, void *stream);

/* Gather m per-RHS single-parity fields (array of m DEVICE pointers given as a HOST array)
 * into the gathered layout, converting precision; and the reverse.
 * Replaces colorSpinorGather / colorSpinorScatter -- reference
 * src/data_format/qcu_data_format_shift.cu:163-205. vh = sites of one parity. */
int qcuGatherMrhs(void *dst, int dst_precision, void *const *src_ptrs, int src_precision,
                  int64_t vh, int n_color, int m_rhs, void *stream);
int qcuScatterMrhs(void *const *dst_ptrs, int dst_precision, const void *src, int src_precision,
                   int64_t vh, int n_color, int m_rhs, void *stream);

/* Precision conversion of n complex numbers.
 * Replaces copyComplexVector_interface -- reference src/data_format/qcu_data_format_shift.cu:141-161. */
int qcuCopyComplexVector(void *dst, int dst_precision, const void *src, int src_precision,
                         int64_t n, void *stream);

/* Multi-RHS BLAS on strided vectors (element i of RHS j at complex offset i*m + j; len
 * complex elements per RHS).  Scalars a, b, c and results are DEVICE arrays of m complex
 * doubles (double2), vectors are in `precision`.  Reductions accumulate in FP64.
 * Replace reference src/qcu_blas/qcu_complex_dotc.cu:20-75, qcu_complex_norm.cu:20-57,
 * qcu_complex_xsay.cu, qcu_complex_xpay.cu, qcu_complex_axpby.cu, qcu_complex_axpbypcz.cu. */
int qcuMrhsDotc(void *res, const void *a, const void *b, int64_t len, int m, int precision,
                void *stream);                                  /* res_j = sum conj(a) b */
int qcuMrhsNorm(double *res, const void *a, int64_t len, int m, int precision,
                void *stream);                                  /* res_j = sqrt(sum |a|^2) */
int qcuMrhsXsay(void *res, const void *x, const void *a, const void *y, int64_t len, int m,
                int precision, void *stream);                   /* res = x - a_j y */
int qcuMrhsXpay(void *res, const void *x, const void *a, const void *y, int64_t len, int m,
                int precision, void *stream);                   /* res = x + a_j y */
int qcuMrhsAxpby(void *res, const void *a, const void *x, const void *b, const void *y,
                 int64_t len, int m, int precision, void *stream); /* res = a_j x + b_j y */
int qcuMrhsAxpbypcz(void *res, const void *a, const void *x, const void *b, const void *y,
                    const void *c, const void *z, int64_t len, int m, int precision,
                    void *stream);                              /* res = a_j x + b_j y + c_j z */
/* qcuMrhsDotc for callers that cannot allocate device memory (their device memory is
 * owned by another allocator, or allocation is not allowed on their code path).  No
 * counterpart in the reference.  Same arguments and result as qcuMrhsDotc; never calls
 * cudaMalloc or cudaFree: its scratch is a fixed 1 MiB device array inside the library
 * (held on every GPU that loads it until exit).  m <= 64, else QCU_ERR_INVALID.  The
 * first call on a device looks up the array's address, so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race. */
int qcuMrhsDotcNoAlloc(void *res, const void *a, const void *b, int64_t len, int m, int precision,
                       void *stream);
/* m-length complex scalar arrays (double2): reference src/qcu_blas/qcu_elementwise_{div,mul,init}.cu */
int qcuElementwiseDiv(void *res, const void *x, const void *y, int m, void *stream);
int qcuElementwiseMul(void *res, const void *x, const void *y, int m, void *stream);
int qcuElementwiseInit(void *res, double re, double im, int m, void *stream);

/* Gauge reorder lexicographic [4][Lt][Lz][Ly][Lx][Nc][Nc] <-> even/odd, on a given lattice
 * (gauge_eo_precondition without a context). */
int qcuGaugeToEO(void *eo, const void *lex, const int L[4], int n_color, int precision, void *stream);
int qcuGaugeFromEO(void *lex, const void *eo, const int L[4], int n_color, int precision, void *stream);
/* Fermion reorder lexicographic [Lt][Lz][Ly][Lx][4][Nc] <-> even/odd [2][Vh][4][Nc] (one RHS).
 * The reference keeps this conversion in its external submodule (absent from its tree);
 * the even/odd convention is the one of include/point/qcu_point.cuh:16-61 (parity
 * (x+y+z+t) mod 2, x = 2*xh + ((p+y+z+t) & 1)). */
int qcuFermionToEO(void *eo, const void *lex, const int L[4], int n_color, int precision, void *stream);
int qcuFermionFromEO(void *lex, const void *eo, const int L[4], int n_color, int precision, void *stream);

/* Site-blocked layout of a multi-RHS half-lattice field (no reference counterpart): the
 * layout the mixed solver keeps its 16-bit vectors in.  Blocks of 32 sites; inside a block
 * the 4 Nc spin-colour rows one after another, each row holding the block's 32 sites with
 * their m right-hand sides innermost:
 *   complex (site n, row r, RHS j) at ((n / 32) 4 Nc + r) 32 m + (n % 32) m + j.
 * A warp reading one row of consecutive sites reads one contiguous run.
 * qcuSiteBlockMrhs reorders gathered [Vh][4][Nc][m] -> blocked (to_blocked = 1) or back
 * (0), not in place; vh must be a multiple of 32.
 * qcuDslashMrhsSiteBlocked is qcuDslashMrhs on blocked in/out: FP16 or BF16, SU(3),
 * m = 8, 12 or 16, vh a multiple of 32. */
int qcuSiteBlockMrhs(void *dst, const void *src, int64_t vh, int n_color, int m_rhs, int precision,
                     int to_blocked, void *stream);
int qcuDslashMrhsSiteBlocked(void *out, const void *in, const void *gauge, const int L[4], int n_color,
                             int m_rhs, int parity, int dagger, double t_sign, int precision, void *stream);

/* Hop kernel selection.
 *   SIMT     one thread per (site, RHS), all colours in registers;
 *   SIMT_CS  one thread per (site, RHS, colour): fewer registers (FP64, large N),
 *            needs n_color * m_rhs <= 256 (else SIMT);
 *   TENSOR   FP16/BF16 storage on the tcgen05 tensor cores with TMEM accumulators, the
 *            MMA operands (projected neighbour spinors, embedded links) written to shared
 *            memory by the CTA's threads, for 2 <= n_color <= 4 and m_rhs <= 32 (else
 *            SIMT);
 *   PACKED16 FP16/BF16 storage, projection and link products in packed 16-bit complex
 *            arithmetic, the 8 hops summed in FP32; 2 <= n_color <= 4, m_rhs >= 2
 *            (else SIMT);
 *   PACKED16_ACC16  as PACKED16, with the 8 hops also summed in FP16 (FP16 storage
 *            only; the accumulation of the reference's half-precision path); less
 *            accurate, so AUTO never picks it;
 *   PACKED16_STAGED as PACKED16, with each site's links staged once per block in shared
 *            memory instead of read by each (site, RHS) thread;
 *   PACKED16_PAIRS  as PACKED16 with two RHS per thread (8-byte neighbour loads, links
 *            shared by the pair), SU(3) with m = 8, 12 or 16 (else PACKED16);
 *   MMA16    FP16/BF16, SU(3), m = 8, 12 or 16: one warp per site, the forward and
 *            backward hop of a direction as one mma.sync m16n8k16 per output spin (link
 *            products in the tensor cores, FP32 accumulation); else as AUTO.  Only an
 *            explicit request selects it: its Schur and residual forms, most of the
 *            solver's hops, are slower than PACKED16_PAIRS's, which the autotuner's
 *            plain-hop timing does not see;
 *   MMA_LINK FP16/BF16, 2 <= n_color <= 8, any m_rhs: one warp per (site, up to 16 RHS; 8
 *            for n_color >= 5), the links as the A operand of mma.sync m16n8k16 and the
 *            projected neighbour half spinors (columns = RHS x half spinor) as B; the
 *            forward and backward hop of a direction are one MMA per 4 RHS (four for
 *            n_color >= 5), link products and the sum of the 8 hops in FP32, the spin
 *            projection the only 16-bit arithmetic.  On a context (the solvers,
 *            start_dslash, mat_Qcu, qcuDslashMrhsContext*) it reads a per-site neighbour
 *            table and hop-link array, and for n_color <= 4 and m_rhs = 4, 8, 12, 16 stages
 *            each site's neighbour, link and epilogue blocks in shared memory with bulk
 *            asynchronous copies (the TMA engine, bounded mbarrier waits);
 *   MMA_LINK_DIRECT  the same kernels without the shared-memory staging (fragment words
 *            loaded straight from global memory): faster where the fields stay in L2;
 *   AUTO     the choice recorded by qcuTuneHop (or loaded from the tuning cache) for
 *            (n_color, m_rhs, precision), else MMA_LINK (n_color >= 5 or m_rhs <= 16),
 *            PACKED16_PAIRS, PACKED16 or SIMT, the first that applies. */
#define QCU_HOP_AUTO 0
#define QCU_HOP_SIMT 1
#define QCU_HOP_TENSOR 2
#define QCU_HOP_SIMT_CS 3
#define QCU_HOP_PACKED16 4
#define QCU_HOP_PACKED16_ACC16 5
#define QCU_HOP_PACKED16_STAGED 6
#define QCU_HOP_PACKED16_PAIRS 7
#define QCU_HOP_MMA16 8
#define QCU_HOP_MMA_LINK 9
#define QCU_HOP_MMA_LINK_DIRECT 10
int qcuSetHopKernel(int kind);
int qcuGetHopKernel(void);

/* Autotuner: times every hop kernel that covers (n_color, m_rhs, precision) on a lattice
 * L with synthetic fields (allocates and frees temporary device buffers), records the
 * fastest for AUTO and, when the environment variable QCU_TUNE_CACHE names a file,
 * appends "n_color m_rhs precision kind microseconds" to it (read back on first use).
 * Returns the chosen QCU_HOP_* kind (>= 1) or a negative status. */
int qcuTuneHop(const int L[4], int n_color, int m_rhs, int precision, void *stream);
/* Recorded choice for AUTO (0 = none recorded). */
int qcuGetTunedHop(int n_color, int m_rhs, int precision);
/* The kind AUTO runs for a shape: the recorded choice, else the static rule. */
int qcuGetAutoHop(int n_color, int m_rhs, int precision);

/* Nonzero if a kernel on the current device gave up a bounded wait (its results are then
 * invalid); synchronises the device.  clear != 0 resets the flag. */
int qcuGetKernelError(int clear);

/* Self-test of the bounded waits of the staged tensor-core hop on the current context
 * (n_color <= 4, m_rhs = 4, 8, 12 or 16): one FP16 hop launch whose shared-memory stages
 * are armed but never filled, so that every wait gives up after limit_cycles clock cycles
 * and the kernel ends with the device error flag set instead of hanging.  *timed_out = 1
 * when the flag was set (the expected outcome); the flag is cleared again and the context
 * stays usable. */
int qcuHopWaitSelfTest(long long limit_cycles, int *timed_out);

/* Device synchronisation helper for bindings that have no CUDA runtime of their own. */
int qcuDeviceSynchronize(void);

/* Arithmetic peak microbenchmarks: the compute ceilings of the hop kernels.  kind:
 *   DFMA  FP64 fused multiply-add on the CUDA cores
 *   FFMA  FP32 fused multiply-add on the CUDA cores
 *   DMMA  FP64 warp MMA (mma.sync m8n8k4, FP64 accumulation)
 *   HMMA  FP16 warp MMA (mma.sync m16n8k16, FP32 accumulation: the link-operand hop's MMA)
 *   BMMA  BF16 warp MMA (same shape)
 * Launches 4 blocks of 256 threads per SM, each thread (FMA) or warp (MMA) issuing `iters`
 * rounds of 8 independent operations, times the second of two launches with CUDA events on
 * `stream` and writes FLOP/s to *flops. */
#define QCU_PEAK_DFMA 1
#define QCU_PEAK_FFMA 2
#define QCU_PEAK_DMMA 3
#define QCU_PEAK_HMMA 4
#define QCU_PEAK_BMMA 5
int qcuPeakRate(int kind, int iters, double *flops, void *stream);

#ifdef __cplusplus
}
#endif
