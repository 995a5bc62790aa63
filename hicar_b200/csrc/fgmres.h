// fgmres.h -- flexible GMRES(m) (k_fgmres.cu).
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace hw {

constexpr int FG_MAXM = 32; // largest restart length

// Device-resident FGMRES state: Hessenberg matrix (column-major, m+1 rows),
// Givens rotations, the rotated right-hand side g, and the stop control.
struct GmresState {
    int m, jdone, it_total, max_iters, status, stop;
    unsigned int ticket;
    int profile;        // 1: kernels ignore stop (per-kernel timing pass)
    double tol_rel, tol_abs, target, bnorm, res0, res, beta, hnext;
    double *hist;
    SolveState *mirror; // its stop flag follows ours (gates the preconditioner kernels)
    double H[(FG_MAXM + 1) * FG_MAXM];
    double cs[FG_MAXM], sn[FG_MAXM], gv[FG_MAXM + 1], y[FG_MAXM];
    double h1[FG_MAXM + 1], h2[FG_MAXM + 1];
};

typedef void (*PrecondFn)(void *ctx, const double *in, double *out, cudaStream_t s);

struct FgmresCtx {
    OpCtx op;
    int m;
    double *x, *b;      // solution (FP64) and right-hand side (FP64)
    double *V, *Z, *W;  // (m+1) basis vectors, m preconditioned vectors, work vector (padded layout)
    double *partials;
    int red_blocks, dot_blocks;
    GmresState *g;
    const double *g_h1, *g_h2, *g_hnext; // device addresses inside *g
    PrecondFn precond;
    void *pctx;
};

void fgmres_reset(GmresState *g, int m, double tol_rel, double tol_abs, int max_iters, double *hist, SolveState *mirror,
                  cudaStream_t s);
void fgmres_set_profile(GmresState *g, int on, cudaStream_t s);
void fgmres_enqueue_restart(const FgmresCtx &f, cudaStream_t s);
void fgmres_enqueue_step(const FgmresCtx &f, int j, cudaStream_t s);
void fgmres_enqueue_finish(const FgmresCtx &f, cudaStream_t s);

}  // namespace hw
