// k_krylov.cu -- the 15-point operator, the Jacobi-Richardson preconditioner and
// the BiCGStab steps of bicgstab_solve (wind_iterative.F90:555-791), templated on
// the Krylov vector type V (double = reference precision, float = FP32 vectors).
//
// Schedule per BiCGStab iteration with n Richardson sweeps (reference order):
//   precond_scale(p -> p^)  [n-1 x (spmv(p^) ; rich)]   spmv_sigma(p^ -> v, <r^,v>)
//   s_precond(s = r - a v ; s^ = D^-1 s) [n-1 x (spmv ; rich)]
//   spmv_dot5(s^ -> t, <t,s> <t,t> <r^,s> <r^,t> <s,s>)   update_xrp(x, r, p)
// Every reduction is FP64 and single pass: each CTA writes one partial per value,
// the last CTA to arrive (atomic ticket) adds the partials in CTA order and runs
// the scalar recurrences of the reference on the device (alpha, omega, beta, the
// recurrence norm, the stopping and breakdown tests), so an iteration needs no
// host synchronisation.  Kernels read the `stop`/`halt` flags and return at once
// when the solve has ended, which lets the host replay a fixed CUDA graph of
// several iterations and read the flag only once per graph.
#include <stdlib.h>

#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "krylov_dev.cuh"

namespace hw {

static int row_grid(const Dims &d, int cap)
{
    long long n = nsegs(d);
    return (int)(n < cap ? n : cap);
}

// ---- y = A x ----
template <typename V>
__global__ void __launch_bounds__(ROWT) spmv_kernel(OpCtx c, const V *__restrict__ x, V *__restrict__ y,
                                                    const SolveState *gate)
{
    if (gated(gate)) return;
    const long long n = nsegs(c.d);
    for (long long s = blockIdx.x; s < n; s += gridDim.x) {
        Seg g = seg_of(c.d, s);
        if (g.ok) y[kidx(c.d, g.i, g.k, g.j)] = (V)spmv_row(c, x, g.i, g.k, g.j);
    }
}

template <typename V>
__global__ void __launch_bounds__(ROWT) spmv_march_kernel(OpCtx c, const V *__restrict__ x, V *__restrict__ y,
                                                          const SolveState *gate)
{
    if (gated(gate)) return;
    march_rows<V>(c, x, [&](long long o, double v) { y[o] = (V)v; });
}

// Operator kernel of a launch (read at every launch, so at graph capture for
// the captured ones): the float4 column-marching kernels for the probed
// operator when nx is a multiple of 4 (the default), the scalar column-marching
// ones when the environment sets HICARW_SPMV_MARCH=1, the row kernels when it
// sets HICARW_SPMV_MARCH=0 (and for the analytic operator).
enum { SPMV_ROW = 0, SPMV_MARCH = 1, SPMV_MARCH4 = 2 };
static int spmv_kind(const OpCtx &c)
{
    if (!c.probed || c.edges) return SPMV_ROW; // decomposed subdomains: the row kernels mask the halo rows
    const char *e = getenv("HICARW_SPMV_MARCH");
    if (e && e[0] == '0') return SPMV_ROW;
    if (e && e[0] == '1') return SPMV_MARCH;
    return march4_ok(c.d) ? SPMV_MARCH4 : SPMV_ROW;
}
// Resident CTAs of a kernel on the whole device (its occupancy at ROWT threads),
// looked up once per kernel.
static int resident_ctas(const void *kernel)
{
    static std::mutex mu;
    static std::vector<std::pair<const void *, int>> cache;
    std::lock_guard<std::mutex> lk(mu);
    for (const auto &e : cache)
        if (e.first == kernel) return e.second;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, ROWT, 0);
    const int n = std::max(1, sms * std::max(1, per_sm));
    cache.emplace_back(kernel, n);
    return n;
}

// One wave of resident CTAs, at most `cap` and at most one warp per work item.
template <typename K>
static int wave_grid(K *kernel, long long warps_needed, int cap)
{
    const int resident = resident_ctas((const void *)kernel);
    const long long n = (warps_needed + MARCH_WARPS - 1) / MARCH_WARPS;
    return (int)std::max<long long>(1, std::min<long long>(n, std::min(cap, resident)));
}

template <typename K>
static int march_grid(K *kernel, const Dims &d, int cap)
{
    return wave_grid(kernel, march_strips(d), cap);
}

template <typename K>
static int march4_grid(K *kernel, const OpCtx &c, int cap)
{
    return wave_grid(kernel, march4_items(c), cap);
}

// ---- the float4 column-marching kernels ----
// Resident CTAs per SM the compiler must allow for (registers): measured at
// 1024x1024x64, four CTAs of 128 threads (128 registers, a few spilled) made
// spmv_sigma 0.99 -> 0.94 ms and spmv_dot5 1.05 -> 1.09 ms, so the
// five-dot kernel keeps three (up to 168 registers, none spilled).
constexpr int M4_CTAS = 4, M4_CTAS_DOT5 = 3;
template <typename V>
__global__ void __launch_bounds__(ROWT, M4_CTAS) spmv_m4_kernel(OpCtx c, const V *__restrict__ x, V *__restrict__ y,
                                                       const SolveState *gate)
{
    if (gated(gate)) return;
    march4_rows<V>(
        c, x,
        [&](long long o, const double (&v)[4]) {
            V t[4];
#pragma unroll
            for (int e = 0; e < 4; e++) t[e] = (V)v[e];
            st4v(y + o, t);
        },
        [&](long long o, double v) { y[o] = (V)v; });
}

template <typename V>
__global__ void __launch_bounds__(ROWT, M4_CTAS) spmv_sigma_m4_kernel(OpCtx c, const V *__restrict__ phat, V *__restrict__ v,
                                                             const V *__restrict__ rhat, SolveState *stt,
                                                             double *partials);
template <typename V>
__global__ void __launch_bounds__(ROWT, M4_CTAS_DOT5) spmv_dot5_m4_kernel(OpCtx c, const V *__restrict__ shat, V *__restrict__ t,
                                                            const V *__restrict__ sv, const V *__restrict__ rhat,
                                                            SolveState *stt, double *hist, double *partials);

template <typename V>
void launch_spmv(const OpCtx &c, const V *x, V *y, const SolveState *gate, cudaStream_t st)
{
    ProfScope ps_("spmv", coef_bytes(c.d) + rows(c.d) * 2.0 * sizeof(V), st);
    const int kind = spmv_kind(c);
    if (kind == SPMV_MARCH4)
        spmv_m4_kernel<V><<<march4_grid(spmv_m4_kernel<V>, c, 148 * 16), ROWT, 0, st>>>(c, x, y, gate);
    else if (kind == SPMV_MARCH)
        spmv_march_kernel<V><<<march_grid(spmv_march_kernel<V>, c.d, 148 * 16), ROWT, 0, st>>>(c, x, y, gate);
    else spmv_kernel<V><<<row_grid(c.d, 148 * 16), ROWT, 0, st>>>(c, x, y, gate);
    count_launch(1);
}

// rho, the initial norm, the target and the first stopping tests (:602-645) from
// the set-up dots <r^,r>, <r,r>, <b,b>.
__device__ __forceinline__ void setup_step(SolveState *stt, double *hist, const double *tot)
{
    stt->rho = tot[0];
    double rn = sqrt(tot[1]);
    stt->rnorm = rn;
    stt->res0 = rn;
    stt->bnorm2 = tot[2];
    stt->target = fmax(stt->tol_abs, stt->tol_rel * sqrt(tot[2])); // :633
    stt->omega = 1.0;
    stt->alpha = 1.0;
    stt->it = 0;
    stt->best_rn = rn;
    stt->best_it = 0;
    hist[0] = rn;
    if (rn <= stt->target) { stt->status = 0; stt->stop = 1; stt->halt = 1; }
    else if (stt->max_iters <= 0) { stt->status = 1; stt->stop = 1; stt->halt = 1; }
}

// ---- setup: r = b - A x0, r^ = r, p = r, <r^,r>, <r,r>, <b,b> (:585-645) ----
// X is the type of the solution (FP64 with FP32 vectors and FP64 lambda).
// restart != 0: a restart of the recurrences from the current solution (the
// true-residual stopping rule): the iteration count, the initial norm and the
// target are kept, the stop flags cleared.
template <typename V, typename X>
__global__ void __launch_bounds__(ROWT) setup_kernel(OpCtx c, const X *__restrict__ x, const V *__restrict__ rhs,
                                                     V *__restrict__ r, V *__restrict__ rhat, V *__restrict__ p,
                                                     SolveState *stt, double *hist, double *partials, int restart)
{
    double acc[3] = {0.0, 0.0, 0.0};
    const long long n = nsegs(c.d);
    for (long long s = blockIdx.x; s < n; s += gridDim.x) {
        Seg g = seg_of(c.d, s);
        if (!g.ok) continue;
        long long o = kidx(c.d, g.i, g.k, g.j);
        double bd = (double)rhs[o];
        V rv = (V)(bd - spmv_row(c, x, g.i, g.k, g.j)); // t = A x0 ; r = 1*b + (-1)*t
        r[o] = rv;
        rhat[o] = rv;
        p[o] = rv;
        if (!owned_row(c.d, c.edges, g.i, g.j)) continue;
        acc[0] += (double)rv * (double)rv; // <r^, r>
        acc[1] += (double)rv * (double)rv; // <r, r>
        acc[2] += bd * bd;                 // <b, b>
    }
    double tot[3];
    if (!grid_reduce<3>(acc, partials, &stt->ticket[0], tot)) return;
    if (stt->dist) { // decomposed solve: the host sums the ranks' totals and applies setup_step
        if (threadIdx.x == 0)
            for (int q = 0; q < 3; q++) stt->dist_tot[q] = tot[q];
        return;
    }
    if (threadIdx.x == 0 && restart) {
        const double rn = sqrt(tot[1]);
        stt->rho = tot[0];
        stt->rnorm = rn;
        stt->omega = 1.0;
        stt->alpha = 1.0;
        stt->best_rn = rn;
        stt->best_it = stt->it;
        stt->status = 1;
        stt->stop = 0;
        stt->halt = 0;
        stt->upd_r = stt->upd_p = 0;
        if (rn <= stt->target) { stt->status = 0; stt->stop = 1; stt->halt = 1; }
        else if (stt->it >= stt->max_iters) { stt->status = 1; stt->stop = 1; stt->halt = 1; }
        return;
    }
    if (threadIdx.x == 0) setup_step(stt, hist, tot);
}

template <typename V, typename X>
void launch_setup(const OpCtx &c, const X *x, const V *rhs, V *r, V *rhat, V *p, SolveState *stt, double *hist,
                  const RedBuf &rb, int restart, cudaStream_t st)
{
    ProfScope ps_("setup", coef_bytes(c.d) + rows(c.d) * (sizeof(X) + 4.0 * sizeof(V)), st);
    setup_kernel<V, X><<<rb.blocks, ROWT, 0, st>>>(c, x, rhs, r, rhat, p, stt, hist, rb.partials, restart);
    count_launch(1);
}

// alpha = rho / sigma (:657-688), on the last CTA of the sigma reduction.
__device__ __forceinline__ void sigma_step(SolveState *stt, double sigma)
{
    stt->sigma = sigma;
    stt->it += 1;
    if (fabs(sigma) < BREAKDOWN_EPS) { stt->status = 2; stt->stop = 1; stt->halt = 1; }
    else stt->alpha = stt->rho / sigma;
}

// omega, rho, beta, the recurrence norm and the stop / breakdown / stall tests
// (:703-783), on the last CTA of the five-dot reduction.
__device__ __forceinline__ void dot5_step(SolveState *stt, double *hist, const double (&tot)[5])
{
    double ts = tot[0], tt = tot[1], rs = tot[2], rt = tot[3], ss = tot[4];
    stt->upd_r = 0;
    stt->upd_p = 0;
    if (tt < BREAKDOWN_EPS) { stt->status = 2; stt->stop = 1; stt->halt = 1; return; } // :737
    double omega = ts / tt;
    double rho_new = rs - omega * rt;
    double rn2 = ss - 2.0 * omega * ts + omega * omega * tt; // :748
    if (rn2 < 0.0) rn2 = 0.0;
    double rn = sqrt(rn2);
    stt->omega = omega;
    stt->rnorm = rn;
    hist[stt->it] = rn;
    if (rn <= stt->target) { stt->status = 0; stt->stop = 1; return; }         // :758 (after x update)
    if (stt->stall_k > 0) { // stall detector: no 1% decrease within stall_k iterations
        if (rn < 0.99 * stt->best_rn) { stt->best_rn = rn; stt->best_it = stt->it; }
        else if (stt->it - stt->best_it >= stt->stall_k) { stt->status = 4; stt->stop = 1; return; }
    }
    if (fabs(omega) < BREAKDOWN_EPS) { stt->status = 2; stt->stop = 1; return; } // :763
    stt->upd_r = 1;
    if (fabs(stt->rho) < BREAKDOWN_EPS) { stt->status = 2; stt->stop = 1; return; } // :774
    stt->beta = (rho_new / stt->rho) * (stt->alpha / omega);
    stt->upd_p = 1;
    stt->rho = rho_new;
    if (stt->it >= stt->max_iters) { stt->status = 1; stt->stop = 1; } // loop ends after this iteration
}

// ---- v = A p^ and sigma = <r^, v> (:657-688) ----
template <typename V>
__global__ void __launch_bounds__(ROWT) spmv_sigma_kernel(OpCtx c, const V *__restrict__ phat, V *__restrict__ v,
                                                          const V *__restrict__ rhat, SolveState *stt, double *partials)
{
    if (gated(stt)) return;
    double acc[1] = {0.0};
    const long long n = nsegs(c.d);
    for (long long s = blockIdx.x; s < n; s += gridDim.x) {
        Seg g = seg_of(c.d, s);
        if (!g.ok) continue;
        long long o = kidx(c.d, g.i, g.k, g.j);
        V vv = (V)spmv_row(c, phat, g.i, g.k, g.j);
        v[o] = vv;
        if (owned_row(c.d, c.edges, g.i, g.j)) acc[0] += (double)rhat[o] * (double)vv;
    }
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &stt->ticket[1], tot)) return;
    if (threadIdx.x == 0) {
        if (stt->dist) stt->dist_tot[0] = tot[0];
        else sigma_step(stt, tot[0]);
    }
}

// The same with column-marching rows (probed operator).
template <typename V>
__global__ void __launch_bounds__(ROWT) spmv_sigma_march_kernel(OpCtx c, const V *__restrict__ phat,
                                                                V *__restrict__ v, const V *__restrict__ rhat,
                                                                SolveState *stt, double *partials)
{
    if (gated(stt)) return;
    double acc[1] = {0.0};
    march_rows<V>(c, phat, [&](long long o, double y) {
        const V vv = (V)y;
        v[o] = vv;
        acc[0] += (double)rhat[o] * (double)vv;
    });
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &stt->ticket[1], tot)) return;
    if (threadIdx.x == 0) sigma_step(stt, tot[0]);
}

// The same with float4 column-marching rows.
template <typename V>
__global__ void __launch_bounds__(ROWT, M4_CTAS) spmv_sigma_m4_kernel(OpCtx c, const V *__restrict__ phat, V *__restrict__ v,
                                                             const V *__restrict__ rhat, SolveState *stt,
                                                             double *partials)
{
    if (gated(stt)) return;
    double acc[1] = {0.0};
    march4_rows<V>(
        c, phat,
        [&](long long o, const double (&y)[4]) {
            V vv[4], rh[4];
#pragma unroll
            for (int e = 0; e < 4; e++) vv[e] = (V)y[e];
            st4v(v + o, vv);
            ld4v(rhat + o, rh);
#pragma unroll
            for (int e = 0; e < 4; e++) acc[0] += (double)rh[e] * (double)vv[e];
        },
        [&](long long o, double y) {
            const V vv = (V)y;
            v[o] = vv;
            acc[0] += (double)rhat[o] * (double)vv;
        });
    double tot[1];
    if (!grid_reduce<1>(acc, partials, &stt->ticket[1], tot)) return;
    if (threadIdx.x == 0) sigma_step(stt, tot[0]);
}

template <typename V>
void launch_spmv_sigma(const OpCtx &c, const V *phat, V *v, const V *rhat, SolveState *stt, const RedBuf &rb,
                       cudaStream_t st)
{
    ProfScope ps_("spmv_sigma", coef_bytes(c.d) + rows(c.d) * 3.0 * sizeof(V), st);
    const int kind = spmv_kind(c);
    if (kind == SPMV_MARCH4)
        spmv_sigma_m4_kernel<V><<<march4_grid(spmv_sigma_m4_kernel<V>, c, rb.blocks), ROWT, 0, st>>>(
            c, phat, v, rhat, stt, rb.partials);
    else if (kind == SPMV_MARCH)
        spmv_sigma_march_kernel<V><<<march_grid(spmv_sigma_march_kernel<V>, c.d, rb.blocks), ROWT, 0, st>>>(
            c, phat, v, rhat, stt, rb.partials);
    else spmv_sigma_kernel<V><<<rb.blocks, ROWT, 0, st>>>(c, phat, v, rhat, stt, rb.partials);
    count_launch(1);
}

// ---- t = A s^ and the packed reduction <t,s> <t,t> <r^,s> <r^,t> <s,s> (:703-783) ----
template <typename V>
__global__ void __launch_bounds__(ROWT) spmv_dot5_kernel(OpCtx c, const V *__restrict__ shat, V *__restrict__ t,
                                                         const V *__restrict__ sv, const V *__restrict__ rhat,
                                                         SolveState *stt, double *hist, double *partials)
{
    if (gated(stt)) return;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const long long n = nsegs(c.d);
    for (long long s = blockIdx.x; s < n; s += gridDim.x) {
        Seg g = seg_of(c.d, s);
        if (!g.ok) continue;
        long long o = kidx(c.d, g.i, g.k, g.j);
        V tv = (V)spmv_row(c, shat, g.i, g.k, g.j);
        t[o] = tv;
        if (!owned_row(c.d, c.edges, g.i, g.j)) continue;
        double td = (double)tv, sd = (double)sv[o], rd = (double)rhat[o];
        acc[0] += td * sd;
        acc[1] += td * td;
        acc[2] += rd * sd;
        acc[3] += rd * td;
        acc[4] += sd * sd;
    }
    double tot[5];
    if (!grid_reduce<5>(acc, partials, &stt->ticket[2], tot)) return;
    if (threadIdx.x == 0) {
        if (stt->dist)
            for (int q = 0; q < 5; q++) stt->dist_tot[q] = tot[q];
        else dot5_step(stt, hist, tot);
    }
}

// The same with column-marching rows (probed operator).
template <typename V>
__global__ void __launch_bounds__(ROWT) spmv_dot5_march_kernel(OpCtx c, const V *__restrict__ shat,
                                                               V *__restrict__ t, const V *__restrict__ sv,
                                                               const V *__restrict__ rhat, SolveState *stt,
                                                               double *hist, double *partials)
{
    if (gated(stt)) return;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    march_rows<V>(c, shat, [&](long long o, double y) {
        const V tv = (V)y;
        t[o] = tv;
        const double td = (double)tv, sd = (double)sv[o], rd = (double)rhat[o];
        acc[0] += td * sd;
        acc[1] += td * td;
        acc[2] += rd * sd;
        acc[3] += rd * td;
        acc[4] += sd * sd;
    });
    double tot[5];
    if (!grid_reduce<5>(acc, partials, &stt->ticket[2], tot)) return;
    if (threadIdx.x == 0) dot5_step(stt, hist, tot);
}

// The same with float4 column-marching rows.
template <typename V>
__global__ void __launch_bounds__(ROWT, M4_CTAS_DOT5) spmv_dot5_m4_kernel(OpCtx c, const V *__restrict__ shat, V *__restrict__ t,
                                                            const V *__restrict__ sv, const V *__restrict__ rhat,
                                                            SolveState *stt, double *hist, double *partials)
{
    if (gated(stt)) return;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    auto add = [&](double td, double sd, double rd) {
        acc[0] += td * sd;
        acc[1] += td * td;
        acc[2] += rd * sd;
        acc[3] += rd * td;
        acc[4] += sd * sd;
    };
    march4_rows<V>(
        c, shat,
        [&](long long o, const double (&y)[4]) {
            V tv[4], s4[4], r4[4];
#pragma unroll
            for (int e = 0; e < 4; e++) tv[e] = (V)y[e];
            st4v(t + o, tv);
            ld4v(sv + o, s4);
            ld4v(rhat + o, r4);
#pragma unroll
            for (int e = 0; e < 4; e++) add((double)tv[e], (double)s4[e], (double)r4[e]);
        },
        [&](long long o, double y) {
            const V tv = (V)y;
            t[o] = tv;
            add((double)tv, (double)sv[o], (double)rhat[o]);
        });
    double tot[5];
    if (!grid_reduce<5>(acc, partials, &stt->ticket[2], tot)) return;
    if (threadIdx.x == 0) dot5_step(stt, hist, tot);
}

template <typename V>
void launch_spmv_dot5(const OpCtx &c, const V *shat, V *t, const V *s, const V *rhat, SolveState *stt, double *hist,
                      const RedBuf &rb, cudaStream_t st)
{
    ProfScope ps_("spmv_dot5", coef_bytes(c.d) + rows(c.d) * 4.0 * sizeof(V), st);
    const int kind = spmv_kind(c);
    if (kind == SPMV_MARCH4)
        spmv_dot5_m4_kernel<V><<<march4_grid(spmv_dot5_m4_kernel<V>, c, rb.blocks), ROWT, 0, st>>>(
            c, shat, t, s, rhat, stt, hist, rb.partials);
    else if (kind == SPMV_MARCH)
        spmv_dot5_march_kernel<V><<<march_grid(spmv_dot5_march_kernel<V>, c.d, rb.blocks), ROWT, 0, st>>>(
            c, shat, t, s, rhat, stt, hist, rb.partials);
    else spmv_dot5_kernel<V><<<rb.blocks, ROWT, 0, st>>>(c, shat, t, s, rhat, stt, hist, rb.partials);
    count_launch(1);
}

// ---- elementwise kernels over the padded vectors (padding stays zero) ----
constexpr int EWT = 256;
static int ew_grid(long long n)
{
    long long b = (n + EWT - 1) / EWT;
    return (int)(b < 148 * 16 ? b : 148 * 16);
}

// out = D^-1 in (sweep 1 of apply_precond, :1289-1297).  The first kernel of an
// iteration also converts a pending `stop` into `halt` for the next iteration.
template <typename V>
__global__ void precond_scale_kernel(long long n, const V *__restrict__ in, V *__restrict__ out,
                                     const V *__restrict__ Dinv, SolveState *gate, int set_halt)
{
    if (gated(gate)) {
        if (set_halt && blockIdx.x == 0 && threadIdx.x == 0) gate->halt = 1;
        return;
    }
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        out[q] = Dinv[q] * in[q];
}

template <typename V>
void launch_precond_scale(const Dims &d, const V *in, V *out, const V *Dinv, SolveState *gate, int set_halt,
                          cudaStream_t st)
{
    ProfScope ps_("precond_scale", rows(d) * 3.0 * sizeof(V), st);
    precond_scale_kernel<V><<<ew_grid(d.npad), EWT, 0, st>>>(d.npad, in, out, Dinv, gate, set_halt);
    count_launch(1);
}

// s = r - alpha v (:690) fused with s^ = D^-1 s (sweep 1 of the second apply)
template <typename V>
__global__ void s_precond_kernel(long long n, const V *__restrict__ r, const V *__restrict__ v, V *__restrict__ s,
                                 V *__restrict__ shat, const V *__restrict__ Dinv, const SolveState *stt)
{
    if (gated(stt)) return;
    const double a = stt->alpha;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        V sv = (V)(1.0 * (double)r[q] + (-a) * (double)v[q]);
        s[q] = sv;
        shat[q] = Dinv[q] * sv;
    }
}

template <typename V>
void launch_s_precond(const Dims &d, const V *r, const V *v, V *s, V *shat, const V *Dinv, SolveState *stt,
                      cudaStream_t st)
{
    ProfScope ps_("s_precond", rows(d) * 5.0 * sizeof(V), st);
    s_precond_kernel<V><<<ew_grid(d.npad), EWT, 0, st>>>(d.npad, r, v, s, shat, Dinv, stt);
    count_launch(1);
}

// out += D^-1 (in - A out) with pres = A out (sweeps 2..n, :1301-1313)
template <typename V>
__global__ void rich_kernel(long long n, const V *__restrict__ in, V *__restrict__ out, const V *__restrict__ pres,
                            const V *__restrict__ Dinv, const SolveState *gate)
{
    if (gated(gate)) return;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        out[q] = out[q] + Dinv[q] * (in[q] - pres[q]);
}

template <typename V>
void launch_rich(const Dims &d, const V *in, V *out, const V *pres, const V *Dinv, const SolveState *gate,
                 cudaStream_t st)
{
    ProfScope ps_("rich", rows(d) * 5.0 * sizeof(V), st);
    rich_kernel<V><<<ew_grid(d.npad), EWT, 0, st>>>(d.npad, in, out, pres, Dinv, gate);
    count_launch(1);
}

// x += alpha p^ + omega s^ (:755); r = s - omega t (:771); p = r + beta (p - omega v) (:781)
template <typename V, typename X>
__global__ void update_xrp_kernel(long long n, X *__restrict__ x, const V *__restrict__ phat, const V *__restrict__ shat,
                                  V *__restrict__ r, const V *__restrict__ s, const V *__restrict__ t, V *__restrict__ p,
                                  const V *__restrict__ v, const SolveState *stt)
{
    if (*(volatile const int *)&stt->halt && !stt->profile) return;
    const double a = stt->alpha, w = stt->omega, b = stt->beta;
    const int ur = stt->upd_r, up = stt->upd_p;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        x[q] = (X)((double)x[q] + a * (double)phat[q] + w * (double)shat[q]);
        if (ur) {
            V rv = (V)(1.0 * (double)s[q] + (-w) * (double)t[q]);
            r[q] = rv;
            if (up) p[q] = (V)((double)rv + b * ((double)p[q] - w * (double)v[q]));
        }
    }
}

template <typename V, typename X>
void launch_update_xrp(const Dims &d, X *x, const V *phat, const V *shat, V *r, const V *s, const V *t, V *p, const V *v,
                       const SolveState *stt, cudaStream_t st)
{
    ProfScope ps_("update_xrp", rows(d) * (2.0 * sizeof(X) + 8.0 * sizeof(V)), st);
    update_xrp_kernel<V, X><<<ew_grid(d.npad), EWT, 0, st>>>(d.npad, x, phat, shat, r, s, t, p, v, stt);
    count_launch(1);
}

// First node of an iteration in schedules whose first kernel is not
// precond_scale: a pending stop becomes halt (no x update in later iterations).
__global__ void iteration_begin_kernel(SolveState *s)
{
    if (s->stop && !s->profile) s->halt = 1;
}

void launch_iteration_begin(SolveState *stt, cudaStream_t st)
{
    iteration_begin_kernel<<<1, 1, 0, st>>>(stt);
    count_launch(1);
}

// ---- decomposed solve: scalar steps on the totals summed over all ranks ----
__global__ void dist_apply_kernel(SolveState *stt, double *hist, int kind, const double *__restrict__ tot)
{
    double t[5];
    for (int q = 0; q < 5; q++) t[q] = q < (kind == 0 ? 3 : kind == 1 ? 1 : 5) ? tot[q] : 0.0;
    if (kind == 0) setup_step(stt, hist, t);
    else if (kind == 1) {
        if (!(stt->stop && !stt->profile)) sigma_step(stt, t[0]);
    } else if (!(stt->stop && !stt->profile)) {
        double t5[5] = {t[0], t[1], t[2], t[3], t[4]};
        dot5_step(stt, hist, t5);
    }
}

void launch_dist_apply(SolveState *stt, double *hist, int kind, const double *tot, cudaStream_t st)
{
    dist_apply_kernel<<<1, 1, 0, st>>>(stt, hist, kind, tot);
    count_launch(1);
}

// zero on the halo cells of the rank-edge sides (the preconditioner's zero halo)
template <typename V>
__global__ void zero_rank_edges_kernel(Dims d, int edges, V *x)
{
    const long long n = (long long)d.mz * d.my;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % d.mz), j = (int)(q / d.mz);
        if (edges & EDGE_W) x[kidx(d, 0, k, j)] = (V)0;
        if (edges & EDGE_E) x[kidx(d, d.mx - 1, k, j)] = (V)0;
    }
    const long long m = (long long)d.mz * d.mx;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < m; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % d.mx), k = (int)(q / d.mx);
        if (edges & EDGE_S) x[kidx(d, i, k, 0)] = (V)0;
        if (edges & EDGE_N) x[kidx(d, i, k, d.my - 1)] = (V)0;
    }
}

template <typename V>
void launch_zero_rank_edges(const Dims &d, int edges, V *x, cudaStream_t st)
{
    if (!edges) return;
    zero_rank_edges_kernel<V><<<64, 256, 0, st>>>(d, edges, x);
    count_launch(1);
}
template void launch_zero_rank_edges<double>(const Dims &, int, double *, cudaStream_t);
template void launch_zero_rank_edges<float>(const Dims &, int, float *, cudaStream_t);

// faces of a decomposed subdomain: side 0 W / 1 E (column i = 1 / nx owned, i = 0 / nx + 1 halo;
// (k, j) in Fortran order), 2 S / 3 N (row j = 1 / ny owned, j = 0 / ny + 1 halo; (i, k) order)
__global__ void face_kernel(Dims d, double *x, int side, double *buf, int unpack)
{
    const bool we = side < 2;
    const long long n = we ? (long long)d.mz * d.my : (long long)d.mx * d.mz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        long long o;
        if (we) {
            const int k = (int)(q % d.mz), j = (int)(q / d.mz);
            const int i = unpack ? (side == 0 ? 0 : d.mx - 1) : (side == 0 ? 1 : d.mx - 2);
            o = kidx(d, i, k, j);
        } else {
            const int i = (int)(q % d.mx), k = (int)(q / d.mx);
            const int j = unpack ? (side == 2 ? 0 : d.my - 1) : (side == 2 ? 1 : d.my - 2);
            o = kidx(d, i, k, j);
        }
        if (unpack) x[o] = buf[q];
        else buf[q] = x[o];
    }
}

void launch_face(const Dims &d, double *x, int side, double *buf, int unpack, cudaStream_t st)
{
    face_kernel<<<64, 256, 0, st>>>(d, x, side, buf, unpack);
    count_launch(1);
}

__global__ void state_reset_kernel(SolveState *s, double tol_rel, double tol_abs, int max_iters, int stall_k)
{
    s->stall_k = stall_k;
    s->best_it = 0;
    s->best_rn = 1e300;
    s->rho = s->alpha = s->omega = s->beta = s->sigma = 0.0;
    s->rnorm = s->res0 = s->bnorm2 = s->target = 0.0;
    s->tol_rel = tol_rel;
    s->tol_abs = tol_abs;
    s->true_res = -1.0;
    s->it = 0;
    s->max_iters = max_iters;
    s->status = 1;
    s->stop = 0;
    s->halt = 0;
    s->upd_r = s->upd_p = 0;
    s->replacements = 0;
    for (int q = 0; q < 8; q++) s->ticket[q] = 0u;
    s->err = 0;
    s->profile = 0;
    s->dist = 0;
}

void launch_state_reset(SolveState *stt, double tol_rel, double tol_abs, int max_iters, int stall_k, cudaStream_t st)
{
    state_reset_kernel<<<1, 1, 0, st>>>(stt, tol_rel, tol_abs, max_iters, stall_k);
    count_launch(1);
}

// ---- FP64 true residual b - A x.  mode 0: norm only (-> true_res);
// mode 1: also r_out = (V)(b - A x) and rho = <r^, r_out> (residual replacement);
// mode 2: restart, r_out = r^ = b - A x, rho = <r, r>, rnorm = ||r||.
template <typename V, typename X>
__global__ void __launch_bounds__(ROWT) true_residual_kernel(OpCtx c, const X *__restrict__ x, const V *__restrict__ rhs,
                                                             V *__restrict__ r_out, V *__restrict__ rhat,
                                                             SolveState *stt, int mode, double *partials)
{
    if (mode == 1 && gated(stt)) return; // a replacement after the solve has stopped changes nothing
    double acc[2] = {0.0, 0.0};
    const long long n = nsegs(c.d);
    for (long long s = blockIdx.x; s < n; s += gridDim.x) {
        Seg g = seg_of(c.d, s);
        if (!g.ok) continue;
        long long o = kidx(c.d, g.i, g.k, g.j);
        if (!owned_row(c.d, c.edges, g.i, g.j)) continue;
        double e = (double)rhs[o] - spmv_row(c, x, g.i, g.k, g.j);
        acc[0] += e * e;
        if (mode >= 1) {
            V ev = (V)e;
            r_out[o] = ev;
            if (mode == 2) {
                rhat[o] = ev;
                acc[1] += (double)ev * (double)ev;
            } else acc[1] += (double)rhat[o] * (double)ev;
        }
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &stt->ticket[3], tot)) return;
    if (threadIdx.x == 0 && stt->dist && mode == 0) { // decomposed: the local sum of squares, summed by the host
        stt->dist_tot[0] = tot[0];
        return;
    }
    if (threadIdx.x == 0) {
        stt->true_res = sqrt(tot[0]);
        if (mode >= 1) {
            stt->rho = tot[1];
            stt->replacements += 1;
        }
        if (mode == 2) stt->rnorm = sqrt(tot[0]);
    }
}

template <typename V, typename X>
void launch_true_residual(const OpCtx &c, const X *x, const V *rhs, V *r_out, const V *rhat, SolveState *stt, int mode,
                          const RedBuf &rb, cudaStream_t st)
{
    ProfScope ps_("true_residual", coef_bytes(c.d) + rows(c.d) * (sizeof(X) + 3.0 * sizeof(V)), st);
    true_residual_kernel<V, X><<<rb.blocks, ROWT, 0, st>>>(c, x, rhs, r_out, const_cast<V *>(rhat), stt, mode, rb.partials);
    count_launch(1);
}

template <typename A, typename B>
__global__ void convert_kernel(long long n, const A *__restrict__ in, B *__restrict__ out)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        out[q] = (B)in[q];
}

template <typename A, typename B>
void launch_convert(long long n, const A *in, B *out, cudaStream_t st)
{
    convert_kernel<A, B><<<ew_grid(n), EWT, 0, st>>>(n, in, out);
    count_launch(1);
}

// ---- explicit instantiations ----
#define INST_V(V)                                                                                                      \
    template void launch_spmv<V>(const OpCtx &, const V *, V *, const SolveState *, cudaStream_t);                    \
    template void launch_precond_scale<V>(const Dims &, const V *, V *, const V *, SolveState *, int, cudaStream_t);  \
    template void launch_s_precond<V>(const Dims &, const V *, const V *, V *, V *, const V *, SolveState *,          \
                                      cudaStream_t);                                                                   \
    template void launch_rich<V>(const Dims &, const V *, V *, const V *, const V *, const SolveState *, cudaStream_t); \
    template void launch_spmv_sigma<V>(const OpCtx &, const V *, V *, const V *, SolveState *, const RedBuf &,        \
                                       cudaStream_t);                                                                  \
    template void launch_spmv_dot5<V>(const OpCtx &, const V *, V *, const V *, const V *, SolveState *, double *,    \
                                      const RedBuf &, cudaStream_t);
INST_V(double)
INST_V(float)
template void launch_update_xrp<double, double>(const Dims &, double *, const double *, const double *, double *,
                                                const double *, const double *, double *, const double *,
                                                const SolveState *, cudaStream_t);
template void launch_update_xrp<float, double>(const Dims &, double *, const float *, const float *, float *,
                                               const float *, const float *, float *, const float *, const SolveState *,
                                               cudaStream_t);
template void launch_setup<double, double>(const OpCtx &, const double *, const double *, double *, double *,
                                           double *, SolveState *, double *, const RedBuf &, int, cudaStream_t);
template void launch_setup<float, double>(const OpCtx &, const double *, const float *, float *, float *, float *,
                                          SolveState *, double *, const RedBuf &, int, cudaStream_t);
template void launch_true_residual<double, double>(const OpCtx &, const double *, const double *, double *,
                                                   const double *, SolveState *, int, const RedBuf &, cudaStream_t);
template void launch_true_residual<float, double>(const OpCtx &, const double *, const float *, float *,
                                                  const float *, SolveState *, int, const RedBuf &, cudaStream_t);
template void launch_convert<double, float>(long long, const double *, float *, cudaStream_t);
template void launch_convert<float, double>(long long, const float *, double *, cudaStream_t);
template void launch_convert<double, double>(long long, const double *, double *, cudaStream_t);

}  // namespace hw
