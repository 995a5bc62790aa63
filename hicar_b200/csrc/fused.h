// fused.h -- FP32 solve schedules (FUSED, MIXED) of the wind solver.
#pragma once
#include "common.cuh"
#include "kernels.h"

struct hicarw_handle;

namespace hw {

struct FusedBufs {
    int ready = 0;
    long long npad = 0;
    float *x = nullptr;     // alias of the FP32 solution vector (owned by the handle)
    double *x64 = nullptr;  // FP64 solution accumulator (MIXED), owned here
};

struct FusedCtx {
    OpCtx op;
    RedBuf rb;
    SolveState *st;
    double *hist;
    const float *div;
    float *x;
    double *x64;
    FusedBufs *fb;
    int replace_every;
    float *r, *rhat, *p, *phat, *v, *s, *shat, *t, *rhs, *Dinv, *pres;
};

int fused_prepare(FusedBufs &fb, const Dims &d, cudaStream_t s);
void fused_free(FusedBufs &fb);
// r0 = b - A x (FP64 residual of the FP64 solution for MIXED), r^ = p = r0.
void fused_setup(const FusedCtx &c, int mixed, cudaStream_t s);
// One BiCGStab iteration of the fused schedule (sweeps Richardson sweeps).
void fused_enqueue_iteration(const FusedCtx &c, int sweeps, int mixed, cudaStream_t s);
// FP64 true residual of the current solution: mode 0 norm only.
void fused_true_residual(const FusedCtx &c, int mode, cudaStream_t s);
// Restart from the FP64 solution: r = r^ = p = b - A x64.
void fused_restart(const FusedCtx &c, cudaStream_t s);

}  // namespace hw

hw::FusedCtx fused_ctx(hicarw_handle *h);
