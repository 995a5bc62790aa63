// k_fused.cu -- FP32 solve schedules of the wind solver.
//
// MIXED precision: Krylov vectors and the operator's coefficients in FP32,
// every inner product and stencil accumulation in FP64, and the solution lambda
// accumulated in FP64 (x64 += alpha p^ + omega s^).  Every `replace_every`
// iterations the recurrence residual is replaced by the FP64 true residual
// b - A x64 (reliable updates of the residual), and p is corrected by the same
// difference, p += (b - A x64) - r, which is the search direction the recurrence
// would have built from the replaced residual.  This is the outer
// iterative-refinement update of lambda: the FP32 Krylov space drives
// corrections, the FP64 solution and residual keep the attainable accuracy at
// FP64 level.
#include "common.cuh"
#include "fused.h"
#include "kernels.h"
#include "krylov_dev.cuh"

namespace hw {

int fused_prepare(FusedBufs &fb, const Dims &d, cudaStream_t s)
{
    if (fb.ready && fb.npad == d.npad) return 0;
    fused_free(fb);
    if (cudaMalloc((void **)&fb.x64, (size_t)d.npad * sizeof(double)) != cudaSuccess) return -1;
    if (cudaMemsetAsync(fb.x64, 0, (size_t)d.npad * sizeof(double), s) != cudaSuccess) return -1;
    fb.npad = d.npad;
    fb.ready = 1;
    return 0;
}

void fused_free(FusedBufs &fb)
{
    if (fb.x64) cudaFree(fb.x64);
    fb.x64 = nullptr;
    fb.ready = 0;
}

void fused_setup(const FusedCtx &c, int mixed, cudaStream_t s)
{
    if (mixed) launch_setup<float, double>(c.op, c.x64, c.rhs, c.r, c.rhat, c.p, c.st, c.hist, c.rb, s);
    else launch_setup<float, float>(c.op, c.x, c.rhs, c.r, c.rhat, c.p, c.st, c.hist, c.rb, s);
}

// r <- (float)(b - A x64);  p <- p + (b - A x64 - r_old);  rho <- <r^, r>.
// Runs only when the iteration just completed is a multiple of `every` and the
// solve goes on (the decision reads device state, uniform over the grid).
__global__ void __launch_bounds__(ROWT) replace_kernel(OpCtx c, const double *__restrict__ x64,
                                                       const float *__restrict__ rhs, float *__restrict__ r,
                                                       float *__restrict__ p, const float *__restrict__ rhat,
                                                       SolveState *stt, int every, double *partials)
{
    if (*(volatile const int *)&stt->stop) return;
    const int it = *(volatile const int *)&stt->it;
    if (every <= 0 || it % every != 0) return;
    double acc[2] = {0.0, 0.0};
    const long long n = nsegs(c.d);
    for (long long sgi = blockIdx.x; sgi < n; sgi += gridDim.x) {
        Seg g = seg_of(c.d, sgi);
        if (!g.ok) continue;
        long long o = kidx(c.d, g.i, g.k, g.j);
        double e = (double)rhs[o] - spmv_row(c, x64, g.i, g.k, g.j);
        double dlt = e - (double)r[o];
        float rn = (float)e;
        r[o] = rn;
        p[o] = (float)((double)p[o] + dlt);
        acc[0] += (double)rhat[o] * (double)rn;
        acc[1] += e * e;
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &stt->ticket[4], tot)) return;
    if (threadIdx.x == 0) {
        stt->rho = tot[0];
        stt->true_res = sqrt(tot[1]);
        stt->replacements += 1;
    }
}

void fused_enqueue_iteration(const FusedCtx &c, int sweeps, int mixed, cudaStream_t s)
{
    const Dims &d = c.op.d;
    SolveState *st = c.st;
    launch_precond_scale<float>(d, c.p, c.phat, c.Dinv, st, 1, s);
    for (int sw = 2; sw <= sweeps; sw++) {
        launch_spmv<float>(c.op, c.phat, c.pres, st, s);
        launch_rich<float>(d, c.p, c.phat, c.pres, c.Dinv, st, s);
    }
    launch_spmv_sigma<float>(c.op, c.phat, c.v, c.rhat, st, c.rb, s);
    launch_s_precond<float>(d, c.r, c.v, c.s, c.shat, c.Dinv, st, s);
    for (int sw = 2; sw <= sweeps; sw++) {
        launch_spmv<float>(c.op, c.shat, c.pres, st, s);
        launch_rich<float>(d, c.s, c.shat, c.pres, c.Dinv, st, s);
    }
    launch_spmv_dot5<float>(c.op, c.shat, c.t, c.s, c.rhat, st, c.hist, c.rb, s);
    if (mixed) {
        launch_update_xrp<float, double>(d, c.x64, c.phat, c.shat, c.r, c.s, c.t, c.p, c.v, st, s);
        replace_kernel<<<c.rb.blocks, ROWT, 0, s>>>(c.op, c.x64, c.rhs, c.r, c.p, c.rhat, st, c.replace_every,
                                                    c.rb.partials);
        count_launch(1);
    } else {
        launch_update_xrp<float, float>(d, c.x, c.phat, c.shat, c.r, c.s, c.t, c.p, c.v, st, s);
    }
}

void fused_true_residual(const FusedCtx &c, int mode, cudaStream_t s)
{
    if (c.x64)
        launch_true_residual<float, double>(c.op, c.x64, c.rhs, nullptr, nullptr, c.st, mode, c.rb, s);
    else
        launch_true_residual<float, float>(c.op, c.x, c.rhs, nullptr, nullptr, c.st, mode, c.rb, s);
}

// Restart: r = r^ = p = b - A x64 with the stop flags cleared.
__global__ void clear_stop_kernel(SolveState *stt)
{
    stt->stop = 0;
    stt->halt = 0;
    stt->status = 1;
}

void fused_restart(const FusedCtx &c, cudaStream_t s)
{
    clear_stop_kernel<<<1, 1, 0, s>>>(c.st);
    count_launch(1);
    // setup recomputes rho, ||r||; keep the original target and iteration count
    launch_true_residual<float, double>(c.op, c.x64, c.rhs, c.r, c.rhat, c.st, 2, c.rb, s);
    cudaMemcpyAsync(c.p, c.r, (size_t)c.op.d.npad * sizeof(float), cudaMemcpyDeviceToDevice, s);
}

}  // namespace hw
