/*
 * qcu.h -- drop-in C interface of the multi-right-hand-side Wilson dslash and
 * BiCGStab solve, implemented for NVIDIA B200 (sm_100a) by libqcu_b200.so.
 *
 * Every declaration here has the signature of the reference's include/qcu.h:1-32
 * (typedefs :7-13, prototypes :14-29), so callers built against the reference
 * (e.g. a ctypes binding) link against this library unchanged.  Semantics follow
 * src/interface.cu:1-142 and src/qcu_interface.cu:1-413 of the reference:
 *
 *   - field pointers are DEVICE pointers owned by the caller;
 *   - gauge layout (even/odd)    [4][2][Lt][Lz][Ly][Lx/2][Nc][Nc] complex, row-major colour;
 *   - fermion layout (even/odd)  [2][Lt][Lz][Ly][Lx/2][Ns=4][Nc] complex
 *     (full lattice for mat_Qcu / qcuInvert, one parity for start_dslash);
 *   - kappa = 1 / (2 (4 + mass));  M = 1 - kappa * D;
 *   - pushBackFermions queues exactly m_rhs (out, in) pairs; every operation
 *     consumes and clears the queue.
 *
 * Errors: the reference aborts the process (errorQcu / CHECK_CUDA / device trap).
 * Here every entry point returns normally and records a status, readable with
 * qcuGetLastStatus() / qcuGetLastError() declared in qcu_b200.h.
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

/* reference include/qcu.h:7-9 -- lattice_size[X, Y, Z, T] of the whole lattice */
typedef struct QcuParam_s {
    int lattice_size[4];
} QcuParam;

/* reference include/qcu.h:11-13 -- process grid; one GPU: {1, 1, 1, 1} */
typedef struct QcuGrid_t {
    int grid_size[4];
} QcuGrid;

/* reference include/qcu.h:14-15, src/interface.cu:20-38 */
void initGridSize(QcuGrid *grid, QcuParam *param, int n_color, int m_rhs, int inputFloatPrecision,
                  int dslashFloatPrecision);
/* reference include/qcu.h:16, src/interface.cu:40-43 */
void pushBackFermions(void *fermionOut, void *fermionIn);
/* reference include/qcu.h:17, src/interface.cu:45-48 */
void loadQcuGauge(void *gauge, int floatPrecision);
/* reference include/qcu.h:18, src/interface.cu:50-53 */
void getDslash(int dslashType, double mass);
/* reference include/qcu.h:19, src/interface.cu:55-58: out[parity] = D in[1 - parity] */
void start_dslash(int parity, int daggerFlag);
/* reference include/qcu.h:20, src/interface.cu:59-62: out = in - kappa D in */
void mat_Qcu(int daggerFlag);
/* reference include/qcu.h:21, src/interface.cu:70-73: even/odd Schur BiCGStab */
void qcuInvert(int max_iteration, double p_max_prec);
/* reference include/qcu.h:22, src/interface.cu:64-68 */
void finalizeQcu();

/* reference include/qcu.h:25-26, src/interface.cu:76-137: lexicographic <-> even/odd gauge */
void gauge_eo_precondition(void *prec_gauge, void *non_prec_gauge, int precision);
void gauge_reverse_eo_precondition(void *non_prec_gauge, void *prec_gauge, int precision);

/* reference include/qcu.h:29, src/interface.cu:139-142 (file format lives in an external
 * submodule absent from the reference tree; see qcu_b200.h for what is supported) */
void read_gauge_from_file(void *gauge, const char *file_path_prefix);

#ifdef __cplusplus
}
#endif
