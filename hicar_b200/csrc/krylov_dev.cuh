// krylov_dev.cuh -- device helpers shared by the Krylov kernel files: one row of
// the 15-point operator (spmv, wind_iterative.F90:813-1027) accumulated in FP64,
// and the single-pass FP64 grid reduction (last-CTA-done ticket).
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace hw {

// Rows of the system, (nx+2)(nz+2)(ny+2), and compulsory coefficient bytes of
// one operator application (15 FP32 coefficients per interior row).
inline double rows(const Dims &d) { return (double)d.mx * d.my * d.mz; }
inline double coef_bytes(const Dims &d) { return 60.0 * (double)d.nx * d.ny * d.nz; }

constexpr int ROWT = 128; // threads per CTA in the row kernels

// ---- one row of y = A x (spmv, :813-1027), accumulated in FP64 ----
template <typename V>
__device__ __forceinline__ double spmv_row(const OpCtx &c, const V *__restrict__ x, int i, int k, int j)
{
    const Dims &d = c.d;
    const long long o = kidx(d, i, k, j);
    if (i == 0 || i == d.mx - 1 || j == 0 || j == d.my - 1) return (double)x[o]; // lateral identity rows
    const long long P = d.P, PL = d.plane, N = d.npad;
    const float *cf = c.coef + o;
    if (c.probed) {
        if (k == 0 || k == d.mz - 1) return (double)x[o]; // ghost-plane identity rows (:873-881)
        // probed 15-point interior (:883-907), reference term order
        double y = (double)cf[CO * N] * (double)x[o - PL - P];
        y += (double)cf[CG * N] * (double)x[o - PL];
        y += (double)cf[CM * N] * (double)x[o - PL + P];
        y += (double)cf[CK * N] * (double)x[o - P - 1];
        y += (double)cf[CC * N] * (double)x[o - P];
        y += (double)cf[CJ * N] * (double)x[o - P + 1];
        y += (double)cf[CE * N] * (double)x[o - 1];
        y += (double)cf[CA * N] * (double)x[o];
        y += (double)cf[CD * N] * (double)x[o + 1];
        y += (double)cf[CI * N] * (double)x[o + P - 1];
        y += (double)cf[CB * N] * (double)x[o + P];
        y += (double)cf[CH * N] * (double)x[o + P + 1];
        y += (double)cf[CN * N] * (double)x[o + PL - P];
        y += (double)cf[CF * N] * (double)x[o + PL];
        y += (double)cf[CL * N] * (double)x[o + PL + P];
        return y;
    }
    const BcCol b = c.bc[(long long)j * d.mx + i];
    if (k == d.mz - 1) return ((double)x[o] - (double)x[o - P]) / b.dztop; // top BC (:950-960)
    if (k == 0) {                                                         // bottom terrain BC (:962-988)
        double y = b.cy * (double)x[o - PL];
        y += b.cy * (double)x[o - PL + P];
        y += b.cx * (double)x[o - 1];
        y += b.m1 * (double)x[o];
        y += (-b.cx) * (double)x[o + 1];
        y += b.cx * (double)x[o + P - 1];
        y += b.p1 * (double)x[o + P];
        y += (-b.cx) * (double)x[o + P + 1];
        y += (-b.cy) * (double)x[o + PL];
        y += (-b.cy) * (double)x[o + PL + P];
        return y;
    }
    // analytic interior: D=E=F=G=1/dx^2, A = -4/dx^2 - B - C (:990-1025)
    const double dx = (double)d.dx;
    const double inv_dx2 = 1.0 / (dx * dx), neg4 = -4.0 * inv_dx2;
    const double bv = (double)cf[CB * N], cv = (double)cf[CC * N];
    const double av = neg4 - bv - cv;
    double y = (double)cf[CO * N] * (double)x[o - PL - P];
    y += inv_dx2 * (double)x[o - PL];
    y += (double)cf[CM * N] * (double)x[o - PL + P];
    y += (double)cf[CK * N] * (double)x[o - P - 1];
    y += cv * (double)x[o - P];
    y += (double)cf[CJ * N] * (double)x[o - P + 1];
    y += inv_dx2 * (double)x[o - 1];
    y += av * (double)x[o];
    y += inv_dx2 * (double)x[o + 1];
    y += (double)cf[CI * N] * (double)x[o + P - 1];
    y += bv * (double)x[o + P];
    y += (double)cf[CH * N] * (double)x[o + P + 1];
    y += (double)cf[CN * N] * (double)x[o + PL - P];
    y += inv_dx2 * (double)x[o + PL];
    y += (double)cf[CL * N] * (double)x[o + PL + P];
    return y;
}

__device__ __forceinline__ bool gated(const SolveState *s)
{
    return s != nullptr && *(volatile const int *)&s->stop && !s->profile;
}

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduce NR partial sums, publish them, and tell the caller whether this CTA
// arrived last.  The last CTA leaves the grid totals in tot[] (thread 0).
template <int NR>
__device__ bool grid_reduce(double (&acc)[NR], double *partials, unsigned int *ticket, double (&tot)[NR])
{
    __shared__ double sh[NR][32];
    __shared__ int last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        double v = warp_sum(acc[r]);
        if (lane == 0) sh[r][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int r = 0; r < NR; r++) {
            double v = lane < nw ? sh[r][lane] : 0.0;
            v = warp_sum(v);
            if (lane == 0) partials[(long long)blockIdx.x * NR + r] = v;
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int r = 0; r < NR; r++) {
        double v = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += __ldcg(&partials[(long long)b * NR + r]);
        v = warp_sum(v);
        __syncthreads();
        if (lane == 0) sh[r][wid] = v;
        __syncthreads();
        if (threadIdx.x < 32) {
            double w = lane < nw ? sh[r][lane] : 0.0;
            w = warp_sum(w);
            if (lane == 0) tot[r] = w;
        }
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// Row-segment iteration: a segment is ROWT consecutive i of one (k, j) line.
struct Seg {
    int i, k, j;
    bool ok;
};
__device__ __forceinline__ Seg seg_of(const Dims &d, long long s)
{
    const int spl = (d.mx + ROWT - 1) / ROWT;
    long long line = s / spl;
    Seg g;
    g.i = (int)(s - line * spl) * ROWT + threadIdx.x;
    g.k = (int)(line % d.mz);
    g.j = (int)(line / d.mz);
    g.ok = g.i < d.mx;
    return g;
}
__host__ __device__ __forceinline__ long long nsegs(const Dims &d)
{
    return (long long)((d.mx + ROWT - 1) / ROWT) * d.mz * d.my;
}

// ---- column-marching rows of y = A x for the probed operator ----
// A warp owns a strip of 32 consecutive columns i of one j row and marches k
// from the bottom ghost plane to the top one.  x at k-1, k, k+1 of its own
// column and of the columns j-1 and j+1 stay in registers (one new load of
// each per level); the i-1 / i+1 neighbours come from the adjacent lanes by
// shuffles, lanes 0 and 31 keeping their own window of the column beyond the
// strip.  Each interior row sums the 15 terms in spmv_row's order (the same
// FP64 value); lateral columns and ghost planes are identity rows.  f(o, y) is
// called for every row of the system, in k order within a column.
constexpr int MARCH_WARPS = 4; // warps per CTA of the marching kernels (blockDim ROWT)

__host__ __device__ __forceinline__ long long march_strips(const Dims &d) { return (long long)((d.mx + 31) / 32) * d.my; }

template <typename V, typename F>
__device__ __forceinline__ void march_rows(const OpCtx &c, const V *__restrict__ x, F &&f)
{
    const Dims &d = c.d;
    const int nbx = (d.mx + 31) / 32;
    const long long nstrips = (long long)nbx * d.my;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const long long P = d.P, PL = d.plane, N = d.npad;
    for (long long w = (long long)blockIdx.x * wpb + wib; w < nstrips; w += (long long)gridDim.x * wpb) {
        const int bx = (int)(w % nbx), j = (int)(w / nbx);
        const int i = bx * 32 + lane;
        const bool live = i < d.mx;
        const long long ob = ((long long)j * d.mz) * P + i + XO; // row k = 0 of the column
        if (j == 0 || j == d.my - 1) { // lateral j rows: identity (warp-uniform)
            if (live)
                for (int k = 0; k < d.mz; k++) f(ob + k * P, (double)x[ob + k * P]);
            continue;
        }
        const bool ident = i == 0 || i == d.mx - 1; // lateral i columns: identity
        const bool west = lane == 0 && live && !ident, east = lane == 31 && live && !ident;
        // windows (k-1, k, k+1) of the own, j-1, j+1, i-1 (lane 0) and i+1 (lane 31) columns
        double c_m = 0.0, c_0 = 0.0, s_m = 0.0, s_0 = 0.0, n_m = 0.0, n_0 = 0.0, w_m = 0.0, w_0 = 0.0, e_m = 0.0,
               e_0 = 0.0;
        if (live) {
            c_m = (double)x[ob];
            c_0 = (double)x[ob + P];
            s_m = (double)x[ob - PL];
            s_0 = (double)x[ob - PL + P];
            n_m = (double)x[ob + PL];
            n_0 = (double)x[ob + PL + P];
            f(ob, c_m); // bottom ghost plane
        }
        if (west) { w_m = (double)x[ob - 1]; w_0 = (double)x[ob - 1 + P]; }
        if (east) { e_m = (double)x[ob + 1]; e_0 = (double)x[ob + 1 + P]; }
        for (int k = 1; k <= d.nz; k++) {
            const long long o = ob + k * P;
            double c_p = 0.0, s_p = 0.0, n_p = 0.0;
            if (live) {
                c_p = (double)x[o + P];
                s_p = (double)x[o - PL + P];
                n_p = (double)x[o + PL + P];
            }
            double w_p = 0.0, e_p = 0.0;
            if (west) w_p = (double)x[o - 1 + P];
            if (east) e_p = (double)x[o + 1 + P];
            // i-1 and i+1 columns from the neighbouring lanes
            const double lm = __shfl_up_sync(0xffffffffu, c_m, 1), l0 = __shfl_up_sync(0xffffffffu, c_0, 1),
                         lp = __shfl_up_sync(0xffffffffu, c_p, 1);
            const double rm = __shfl_down_sync(0xffffffffu, c_m, 1), r0 = __shfl_down_sync(0xffffffffu, c_0, 1),
                         rp = __shfl_down_sync(0xffffffffu, c_p, 1);
            const double xwm = lane == 0 ? w_m : lm, xw0 = lane == 0 ? w_0 : l0, xwp = lane == 0 ? w_p : lp;
            const double xem = lane == 31 ? e_m : rm, xe0 = lane == 31 ? e_0 : r0, xep = lane == 31 ? e_p : rp;
            if (live) {
                double y;
                if (ident) {
                    y = c_0;
                } else { // probed 15-point interior (:883-907), reference term order
                    const float *cf = c.coef + o;
                    y = (double)cf[CO * N] * s_m;
                    y += (double)cf[CG * N] * s_0;
                    y += (double)cf[CM * N] * s_p;
                    y += (double)cf[CK * N] * xwm;
                    y += (double)cf[CC * N] * c_m;
                    y += (double)cf[CJ * N] * xem;
                    y += (double)cf[CE * N] * xw0;
                    y += (double)cf[CA * N] * c_0;
                    y += (double)cf[CD * N] * xe0;
                    y += (double)cf[CI * N] * xwp;
                    y += (double)cf[CB * N] * c_p;
                    y += (double)cf[CH * N] * xep;
                    y += (double)cf[CN * N] * n_m;
                    y += (double)cf[CF * N] * n_0;
                    y += (double)cf[CL * N] * n_p;
                }
                f(o, y);
            }
            c_m = c_0; c_0 = c_p;
            s_m = s_0; s_0 = s_p;
            n_m = n_0; n_0 = n_p;
            w_m = w_0; w_0 = w_p;
            e_m = e_0; e_0 = e_p;
        }
        if (live) f(ob + (long long)(d.mz - 1) * P, c_0); // top ghost plane (c_0 = x at k = nz + 1)
    }
}


}  // namespace hw
