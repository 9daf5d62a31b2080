// blas.h -- internal host API of the multi-RHS BLAS and fused BiCGStab steps.
#pragma once

#include "common.cuh"
#include "reduce.cuh"
#include "workspace.h"

namespace qcub {

enum AxpyOp : int { OP_XSAY = 0, OP_XPAY = 1, OP_AXPBY = 2, OP_AXPBYPCZ = 3 };

int check_mrhs(int64_t len, int m);

// res: device double2[m]
int mrhs_dotc(double2* res, const void* a, const void* b, int64_t len, int m, int prec,
              const Scratch& ws, cudaStream_t st);
// fin = FIN_NORM writes sqrt into res[m]; FIN_RNORM writes |a|^2 into sc->rnorm2
int mrhs_norm(double* res, const void* a, int64_t len, int m, int prec, const Scratch& ws,
              cudaStream_t st, int fin = FIN_NORM, BicgScalars* sc = nullptr);
// op: OP_XSAY, OP_XPAY, OP_AXPBY, OP_AXPBYPCZ (see blas_impl.cuh); scalars device double2[m]
int mrhs_axpy(int op, void* res, const void* a, const void* x, const void* b, const void* y,
              const void* c, const void* z, int64_t len, int m, int prec, cudaStream_t st);
// op: 0 div, 1 mul, 2 init(re, im)
int elementwise(int op, void* res, const void* x, const void* y, int m, double re, double im,
                cudaStream_t st);

enum BicgStep : int { STEP_INIT = 0, STEP_S = 1, STEP_XR = 2, STEP_P = 3 };

struct BicgStepArgs {
    void* src = nullptr;   // INIT: b'
    void* r0 = nullptr;
    void* r = nullptr;
    void* p = nullptr;
    void* v = nullptr;
    void* s = nullptr;
    void* t = nullptr;
    void* x = nullptr;     // solution accumulator (FP64 plain, FP32 sloppy)
    BicgScalars* sc = nullptr;
    Scratch ws;
    int64_t len = 0;       // complex elements per RHS
    int m = 0;
};

// prec: vector precision; x_prec: accumulator precision (FP64 with FP64, else FP32).
int bicg_step(int step, int prec, int x_prec, const BicgStepArgs& a, cudaStream_t st);

// Mixed precision (gated on sc->gate unless init): x64 += e / scale, e = 0
int mp_accum(void* x64, void* e, BicgScalars* sc, int64_t len, int m, cudaStream_t st);
// rs = scale * r64 (sloppy), p/r0 reset or rescaled, rho = <r0s, rs>
int mp_load(int prec, void* rs, void* ps, void* r0s, const void* r64, BicgScalars* sc, int64_t len,
            int m, int init, const Scratch& ws, cudaStream_t st);
// convergence of the FP64 true residual, new scales
int mp_update(BicgScalars* sc, int m, int init, cudaStream_t st);

}  // namespace qcub
