// k_fgmres.cu -- flexible GMRES(m) for the wind solver's system A lambda = b.
//
// Right-preconditioned flexible GMRES (Saad 1993): the preconditioned vectors
// z_j = M_j^-1 v_j are stored, so the preconditioner may change from step to
// step (a learned, non-linear M is allowed).  Every inner product and the
// Hessenberg / Givens recurrences run in FP64 on the device; the Arnoldi basis
// is orthogonalised by classical Gram-Schmidt applied twice (CGS2).  One restart
// cycle (m steps + the solution update) is one CUDA graph; kernels of steps after
// convergence return at once, and the host reads the stop flag once per cycle.
//
// Per step j (v_j has unit norm):
//   z_j = M^-1 v_j                         (preconditioner, caller-supplied launches)
//   w = A z_j                              fgmres_spmv
//   h1_i = <v_i, w>, i <= j                fgmres_dots + fgmres_fin1
//   w -= sum h1_i v_i                      fgmres_axpy
//   h2_i = <v_i, w>, |w|^2                 fgmres_dots + fgmres_fin2 (Givens, residual estimate, stop)
//   v_{j+1} = (w - sum h2_i v_i) / h_{j+1,j}  fgmres_axpy
// After the cycle: y = H^-1 g (back substitution), x += Z y.
#include <math.h>

#include "common.cuh"
#include "fgmres.h"
#include "kernels.h"
#include "krylov_dev.cuh"

namespace hw {

constexpr int FGT = 256;

__device__ __forceinline__ bool fg_gated(const GmresState *g)
{
    return *(volatile const int *)&g->stop != 0 && !g->profile;
}

// w = A z (probed or analytic operator, FP64)
__global__ void __launch_bounds__(ROWT) fgmres_spmv_kernel(OpCtx c, const double *__restrict__ z,
                                                           double *__restrict__ w, const GmresState *g)
{
    if (fg_gated(g)) return;
    const long long n = nsegs(c.d);
    for (long long s = blockIdx.x; s < n; s += gridDim.x) {
        Seg sg = seg_of(c.d, s);
        if (sg.ok) w[kidx(c.d, sg.i, sg.k, sg.j)] = spmv_row(c, z, sg.i, sg.k, sg.j);
    }
}

// partial[i * B + b] = sum over this CTA's chunk of V_i . w   (blockIdx.y = i < nv),
// slice nv (when with_norm) = w . w
__global__ void __launch_bounds__(FGT) fgmres_dots_kernel(long long n, const double *__restrict__ V, long long ldv,
                                                          const double *__restrict__ w, int nv, int with_norm,
                                                          double *__restrict__ partial, const GmresState *g)
{
    if (fg_gated(g)) return;
    const int i = blockIdx.y;
    const double *a = i < nv ? V + (long long)i * ldv : w;
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        acc += a[q] * w[q];
    acc = warp_sum(acc);
    __shared__ double sh[FGT / 32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < FGT / 32; q++) s += sh[q];
        partial[(long long)i * gridDim.x + blockIdx.x] = s;
    }
    (void)with_norm;
}

// w = w - sum_{i < nv} coef_i V_i ; optionally out = (that) / scale (coef, scale from the state)
__global__ void __launch_bounds__(FGT) fgmres_axpy_kernel(long long n, const double *__restrict__ V, long long ldv,
                                                          double *__restrict__ w, int nv, const double *__restrict__ coef,
                                                          double *__restrict__ out, const double *__restrict__ scale,
                                                          const GmresState *g)
{
    if (fg_gated(g)) return;
    const double inv = scale ? 1.0 / *scale : 1.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        double v = w[q];
        for (int i = 0; i < nv; i++) v -= coef[i] * V[(long long)i * ldv + q];
        if (out) out[q] = v * inv;
        else w[q] = v;
    }
}

// sum the per-CTA partials of the first pass: h1[i] (i <= j)
__global__ void fgmres_fin1_kernel(const double *__restrict__ partial, int nb, int nv, GmresState *g)
{
    if (fg_gated(g)) return;
    int i = threadIdx.x;
    if (i < nv) {
        double s = 0.0;
        for (int b = 0; b < nb; b++) s += partial[(long long)i * nb + b];
        g->h1[i] = s;
    }
}

// second pass: h2, the Hessenberg column j, its Givens rotation, the residual
// estimate |g_{j+1}| and the stop test.
__global__ void fgmres_fin2_kernel(const double *__restrict__ partial, int nb, int j, GmresState *g)
{
    if (fg_gated(g)) return;
    __shared__ double sh2[FG_MAXM + 2];
    const int nv = j + 1;
    int i = threadIdx.x;
    if (i <= nv) { // slices 0..j: <v_i, w>, slice nv: <w, w>
        double s = 0.0;
        for (int b = 0; b < nb; b++) s += partial[(long long)i * nb + b];
        sh2[i] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int m = g->m;
    double ww = sh2[nv], corr = 0.0;
    double *H = g->H + (long long)j * (m + 1); // column j
    for (int q = 0; q < nv; q++) {
        g->h2[q] = sh2[q];
        H[q] = g->h1[q] + sh2[q];
        corr += sh2[q] * sh2[q];
    }
    double hn2 = ww - corr;
    double hn = hn2 > 0.0 ? sqrt(hn2) : 0.0;
    H[nv] = hn;
    g->hnext = hn;
    // apply the previous rotations to column j, then form the new one
    for (int q = 0; q < j; q++) {
        double a = H[q], b = H[q + 1];
        H[q] = g->cs[q] * a + g->sn[q] * b;
        H[q + 1] = -g->sn[q] * a + g->cs[q] * b;
    }
    double a = H[j], b = H[nv];
    double r = sqrt(a * a + b * b);
    double cs = r > 0.0 ? a / r : 1.0, sn = r > 0.0 ? b / r : 0.0;
    g->cs[j] = cs;
    g->sn[j] = sn;
    H[j] = r;
    H[nv] = 0.0;
    g->gv[nv] = -sn * g->gv[j];
    g->gv[j] = cs * g->gv[j];
    g->jdone = nv;
    g->it_total += 1;
    double res = fabs(g->gv[nv]);
    g->res = res;
    if (g->hist && g->it_total <= g->max_iters) g->hist[g->it_total] = res;
    if (res <= g->target || hn < 1e-300 || g->it_total >= g->max_iters) {
        g->stop = 1;
        g->status = res <= g->target ? 0 : (hn < 1e-300 ? 2 : 1);
        if (g->mirror) g->mirror->stop = 1;
    }
}

// y = H(0:jdone, 0:jdone)^-1 g (back substitution on the rotated, upper-triangular H)
__global__ void fgmres_solve_kernel(GmresState *g)
{
    const int m = g->m, n = g->jdone;
    for (int i = n - 1; i >= 0; i--) {
        double s = g->gv[i];
        for (int q = i + 1; q < n; q++) s -= g->H[(long long)q * (m + 1) + i] * g->y[q];
        double d = g->H[(long long)i * (m + 1) + i];
        g->y[i] = d != 0.0 ? s / d : 0.0;
    }
}

// x += sum_{i < jdone} y_i Z_i
__global__ void __launch_bounds__(FGT) fgmres_update_kernel(long long n, const double *__restrict__ Z, long long ldz,
                                                            double *__restrict__ x, const GmresState *g)
{
    const int nv = g->jdone;
    const double *y = g->y;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        double v = x[q];
        for (int i = 0; i < nv; i++) v += y[i] * Z[(long long)i * ldz + q];
        x[q] = v;
    }
}

// restart: v_0 = (b - A x) / beta, g = (beta, 0, ...), rotations cleared
__global__ void __launch_bounds__(ROWT) fgmres_residual_kernel(OpCtx c, const double *__restrict__ x,
                                                               const double *__restrict__ b, double *__restrict__ v0,
                                                               double *partials, GmresState *g)
{
    double acc[2] = {0.0, 0.0};
    const long long n = nsegs(c.d);
    for (long long s = blockIdx.x; s < n; s += gridDim.x) {
        Seg sg = seg_of(c.d, s);
        if (!sg.ok) continue;
        long long o = kidx(c.d, sg.i, sg.k, sg.j);
        double bv = b[o];
        double e = bv - spmv_row(c, x, sg.i, sg.k, sg.j);
        v0[o] = e;
        acc[0] += e * e;
        acc[1] += bv * bv;
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &g->ticket, tot)) return;
    if (threadIdx.x == 0) {
        double beta = sqrt(tot[0]);
        g->beta = beta;
        g->jdone = 0;
        for (int q = 0; q <= g->m; q++) g->gv[q] = 0.0;
        g->gv[0] = beta;
        if (g->it_total == 0) {
            g->bnorm = sqrt(tot[1]);
            g->res0 = beta;
            g->target = fmax(g->tol_abs, g->tol_rel * g->bnorm);
            if (g->hist) g->hist[0] = beta;
        }
        g->res = beta;
        g->stop = 0;
        if (beta <= g->target) { g->stop = 1; g->status = 0; }
        if (g->mirror) g->mirror->stop = g->stop;
    }
}

__global__ void __launch_bounds__(FGT) fgmres_scale_kernel(long long n, double *__restrict__ v, const GmresState *g)
{
    if (fg_gated(g)) return;
    const double inv = 1.0 / g->beta;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        v[q] *= inv;
}

__global__ void fgmres_reset_kernel(GmresState *g, int m, double tol_rel, double tol_abs, int max_iters, double *hist,
                                    SolveState *mirror)
{
    g->mirror = mirror;
    if (mirror) { mirror->stop = 0; mirror->halt = 0; mirror->profile = 0; }
    g->m = m;
    g->tol_rel = tol_rel;
    g->tol_abs = tol_abs;
    g->max_iters = max_iters;
    g->it_total = 0;
    g->status = 1;
    g->stop = 0;
    g->jdone = 0;
    g->ticket = 0u;
    g->profile = 0;
    g->hist = hist;
}

__global__ void fgmres_profile_kernel(GmresState *g, int on)
{
    g->profile = on;
    g->stop = 0;
    g->it_total = 0;
}

// ---------------------------------------------------------------------------
static int ew_blocks(long long n)
{
    long long b = (n + FGT - 1) / FGT;
    return (int)(b < 148 * 8 ? b : 148 * 8);
}

void fgmres_reset(GmresState *g, int m, double tol_rel, double tol_abs, int max_iters, double *hist, SolveState *mirror,
                  cudaStream_t s)
{
    fgmres_reset_kernel<<<1, 1, 0, s>>>(g, m, tol_rel, tol_abs, max_iters, hist, mirror);
    count_launch(1);
}

void fgmres_set_profile(GmresState *g, int on, cudaStream_t s)
{
    fgmres_profile_kernel<<<1, 1, 0, s>>>(g, on);
    count_launch(1);
}

void fgmres_enqueue_restart(const FgmresCtx &f, cudaStream_t s)
{
    const Dims &d = f.op.d;
    {
        ProfScope ps_("fgmres_residual", coef_bytes(d) + rows(d) * 24.0, s);
        fgmres_residual_kernel<<<f.red_blocks, ROWT, 0, s>>>(f.op, f.x, f.b, f.V, f.partials, f.g);
        count_launch(1);
    }
    ProfScope ps_("fgmres_scale", rows(d) * 16.0, s);
    fgmres_scale_kernel<<<ew_blocks(d.npad), FGT, 0, s>>>(d.npad, f.V, f.g);
    count_launch(1);
}

void fgmres_enqueue_step(const FgmresCtx &f, int j, cudaStream_t s)
{
    const Dims &d = f.op.d;
    const long long n = d.npad, ld = d.npad;
    double *vj = f.V + (long long)j * ld, *zj = f.Z + (long long)j * ld;
    f.precond(f.pctx, vj, zj, s); // z_j = M^-1 v_j
    {
        ProfScope ps_("fgmres_spmv", coef_bytes(d) + rows(d) * 16.0, s);
        fgmres_spmv_kernel<<<148 * 16, ROWT, 0, s>>>(f.op, zj, f.W, f.g);
        count_launch(1);
    }
    const int nv = j + 1, nb = f.dot_blocks;
    {
        ProfScope ps_("fgmres_dots", rows(d) * 8.0 * (nv + 1), s);
        fgmres_dots_kernel<<<dim3(nb, nv), FGT, 0, s>>>(n, f.V, ld, f.W, nv, 0, f.partials, f.g);
        count_launch(1);
    }
    fgmres_fin1_kernel<<<1, FG_MAXM + 2, 0, s>>>(f.partials, nb, nv, f.g);
    count_launch(1);
    {
        ProfScope ps_("fgmres_axpy", rows(d) * 8.0 * (nv + 2), s);
        fgmres_axpy_kernel<<<ew_blocks(n), FGT, 0, s>>>(n, f.V, ld, f.W, nv, f.g_h1, nullptr, nullptr, f.g);
        count_launch(1);
    }
    {
        ProfScope ps_("fgmres_dots", rows(d) * 8.0 * (nv + 2), s);
        fgmres_dots_kernel<<<dim3(nb, nv + 1), FGT, 0, s>>>(n, f.V, ld, f.W, nv, 1, f.partials, f.g);
        count_launch(1);
    }
    fgmres_fin2_kernel<<<1, FG_MAXM + 2, 0, s>>>(f.partials, nb, j, f.g);
    count_launch(1);
    {
        ProfScope ps_("fgmres_axpy", rows(d) * 8.0 * (nv + 2), s);
        fgmres_axpy_kernel<<<ew_blocks(n), FGT, 0, s>>>(n, f.V, ld, f.W, nv, f.g_h2, f.V + (long long)(j + 1) * ld,
                                                        f.g_hnext, f.g);
        count_launch(1);
    }
}

void fgmres_enqueue_finish(const FgmresCtx &f, cudaStream_t s)
{
    const Dims &d = f.op.d;
    fgmres_solve_kernel<<<1, 1, 0, s>>>(f.g);
    count_launch(1);
    ProfScope ps_("fgmres_update", rows(d) * 8.0 * (f.m + 2), s);
    fgmres_update_kernel<<<ew_blocks(d.npad), FGT, 0, s>>>(d.npad, f.Z, d.npad, f.x, f.g);
    count_launch(1);
}

}  // namespace hw
