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

namespace hw {

// ---- float4 column-marching rows of y = A x (probed operator, nx % 4 == 0) ----
// A lane owns four consecutive interior columns i0 .. i0+3 (i0 = 1 + 4g: a
// 16-byte aligned group in the padded layout), a warp a strip of 128 columns
// of one j row, and it marches k upwards over a chunk of at most M4_KC levels
// (OpCtx::kc when set: a tuning knob).
// Every coefficient and vector row is read with one 16-byte load per lane (a
// 512-byte segment per warp); x at k-1, k, k+1 of the own row and of the rows
// j-1 and j+1 stays in registers (three new loads per level); the columns
// i0-1 and i0+4 come from the neighbouring lanes by shuffles, and the lanes at
// the ends of a strip load their outer column themselves.  Each interior row
// sums its 15 terms in spmv_row's order, in FP64 (the same values bit for
// bit).  Identity rows: the lateral j rows, the ghost planes, and the lateral
// columns i = 0 and i = mx - 1 (a scalar row, done by the strip's first lane
// and by the lane of the last group).  Work items (j, strip, level chunk) are
// ordered j fastest, so that warps running at the same time share the x rows
// j +- 1 through L2.  f4(o, y[4]) receives a group's four values at the
// offset of its first element, f1(o, y) a scalar row.
constexpr int M4_KC = 16;

__device__ __forceinline__ void ld4v(const float *__restrict__ p, float (&o)[4])
{
    const float4 t = *reinterpret_cast<const float4 *>(p);
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
__device__ __forceinline__ void ld4v(const double *__restrict__ p, double (&o)[4])
{
    const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void st4v(float *__restrict__ p, const float (&v)[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4v(double *__restrict__ p, const double (&v)[4])
{
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(v[2], v[3]);
}

__host__ __device__ __forceinline__ bool march4_ok(const Dims &d) { return d.nx % 4 == 0 && d.nx >= 4; }
__host__ __device__ __forceinline__ int march4_kc(const OpCtx &c) { return c.kc > 0 ? c.kc : M4_KC; }
__host__ __device__ __forceinline__ long long march4_items(const OpCtx &c)
{
    const Dims &d = c.d;
    const int KC = march4_kc(c), G = d.nx / 4, nsx = (G + 31) / 32, nkc = (d.mz + KC - 1) / KC;
    return (long long)d.my * nsx * nkc;
}

template <typename V, typename F4, typename F1>
__device__ __forceinline__ void march4_rows(const OpCtx &c, const V *__restrict__ x, F4 &&f4, F1 &&f1)
{
    const Dims &d = c.d;
    const int KC = march4_kc(c), G = d.nx / 4, nsx = (G + 31) / 32, nkc = (d.mz + KC - 1) / KC;
    const long long items = (long long)d.my * nsx * nkc;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const long long P = d.P, PL = d.plane, N = d.npad;
    for (long long w = (long long)blockIdx.x * wpb + wib; w < items; w += (long long)gridDim.x * wpb) {
        const int j = (int)(w % d.my);
        const long long rest = w / d.my;
        const int bx = (int)(rest % nsx), kc = (int)(rest / nsx);
        const int g = bx * 32 + lane;
        const bool live = g < G;
        const int k0 = kc * KC, k1 = min(k0 + KC, d.mz) - 1;
        const long long ob = (long long)j * PL + 1 + XO + 4LL * g; // group start at k = 0
        const long long oc = (long long)j * PL + XO;                // column i = 0 at k = 0
        const bool first = live && g == 0, lastg = live && g == G - 1;
        // lateral columns i = 0 and i = mx - 1: identity rows
        if (first)
            for (int k = k0; k <= k1; k++) f1(oc + k * P, (double)x[oc + k * P]);
        if (lastg)
            for (int k = k0; k <= k1; k++) f1(oc + (d.mx - 1) + k * P, (double)x[oc + (d.mx - 1) + k * P]);
        if (j == 0 || j == d.my - 1) { // lateral j rows: identity (warp-uniform)
            if (live)
                for (int k = k0; k <= k1; k++) {
                    V xv[4];
                    ld4v(x + ob + k * P, xv);
                    const double y[4] = {(double)xv[0], (double)xv[1], (double)xv[2], (double)xv[3]};
                    f4(ob + k * P, y);
                }
            continue;
        }
        const bool west = live && lane == 0, east = live && (lane == 31 || g == G - 1);
        // windows at k-1 (m), k (0) of the own row (c), the rows j-1 (s) and j+1 (n); the outer columns
        V c_m[4] = {}, c_0[4] = {}, s_m[4] = {}, s_0[4] = {}, n_m[4] = {}, n_0[4] = {};
        V w_m = 0, w_0 = 0, e_m = 0, e_0 = 0;
        if (live) {
            ld4v(x + ob + k0 * P, c_0);
            ld4v(x + ob - PL + k0 * P, s_0);
            ld4v(x + ob + PL + k0 * P, n_0);
            if (k0 > 0) {
                ld4v(x + ob + (k0 - 1) * P, c_m);
                ld4v(x + ob - PL + (k0 - 1) * P, s_m);
                ld4v(x + ob + PL + (k0 - 1) * P, n_m);
            }
        }
        if (west) { w_0 = x[ob - 1 + k0 * P]; if (k0 > 0) w_m = x[ob - 1 + (k0 - 1) * P]; }
        if (east) { e_0 = x[ob + 4 + k0 * P]; if (k0 > 0) e_m = x[ob + 4 + (k0 - 1) * P]; }
        for (int k = k0; k <= k1; k++) {
            const long long o = ob + k * P;
            const bool interior = k >= 1 && k <= d.nz;
            V c_p[4] = {}, s_p[4] = {}, n_p[4] = {};
            V w_p = 0, e_p = 0;
            float cf[15][4];
            if (live && k + 1 < d.mz) {
                ld4v(x + o + P, c_p);
                ld4v(x + o - PL + P, s_p);
                ld4v(x + o + PL + P, n_p);
                if (west) w_p = x[o - 1 + P];
                if (east) e_p = x[o + 4 + P];
            }
            if (live && interior) {
#pragma unroll
                for (int q = 0; q < 15; q++) {
                    const float4 t = __ldg(reinterpret_cast<const float4 *>(c.coef + q * N + o));
                    cf[q][0] = t.x; cf[q][1] = t.y; cf[q][2] = t.z; cf[q][3] = t.w;
                }
            }
            // the columns i0-1 (element 0's west) and i0+4 (element 3's east) from the neighbouring lanes
            const V lm = __shfl_up_sync(0xffffffffu, c_m[3], 1), l0 = __shfl_up_sync(0xffffffffu, c_0[3], 1),
                    lp = __shfl_up_sync(0xffffffffu, c_p[3], 1);
            const V rm = __shfl_down_sync(0xffffffffu, c_m[0], 1), r0 = __shfl_down_sync(0xffffffffu, c_0[0], 1),
                    rp = __shfl_down_sync(0xffffffffu, c_p[0], 1);
            if (live) {
                double y[4];
                if (!interior) {
#pragma unroll
                    for (int e = 0; e < 4; e++) y[e] = (double)c_0[e];
                } else {
                    const V wm = west ? w_m : lm, w0 = west ? w_0 : l0, wp = west ? w_p : lp;
                    const V em = east ? e_m : rm, e0 = east ? e_0 : r0, ep = east ? e_p : rp;
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const double xwm = e > 0 ? (double)c_m[e - 1] : (double)wm;
                        const double xw0 = e > 0 ? (double)c_0[e - 1] : (double)w0;
                        const double xwp = e > 0 ? (double)c_p[e - 1] : (double)wp;
                        const double xem = e < 3 ? (double)c_m[e + 1] : (double)em;
                        const double xe0 = e < 3 ? (double)c_0[e + 1] : (double)e0;
                        const double xep = e < 3 ? (double)c_p[e + 1] : (double)ep;
                        // probed 15-point interior (:883-907), reference term order
                        double v = (double)cf[CO][e] * (double)s_m[e];
                        v += (double)cf[CG][e] * (double)s_0[e];
                        v += (double)cf[CM][e] * (double)s_p[e];
                        v += (double)cf[CK][e] * xwm;
                        v += (double)cf[CC][e] * (double)c_m[e];
                        v += (double)cf[CJ][e] * xem;
                        v += (double)cf[CE][e] * xw0;
                        v += (double)cf[CA][e] * (double)c_0[e];
                        v += (double)cf[CD][e] * xe0;
                        v += (double)cf[CI][e] * xwp;
                        v += (double)cf[CB][e] * (double)c_p[e];
                        v += (double)cf[CH][e] * xep;
                        v += (double)cf[CN][e] * (double)n_m[e];
                        v += (double)cf[CF][e] * (double)n_0[e];
                        v += (double)cf[CL][e] * (double)n_p[e];
                        y[e] = v;
                    }
                }
                f4(o, y);
            }
#pragma unroll
            for (int e = 0; e < 4; e++) {
                c_m[e] = c_0[e]; c_0[e] = c_p[e];
                s_m[e] = s_0[e]; s_0[e] = s_p[e];
                n_m[e] = n_0[e]; n_0[e] = n_p[e];
            }
            w_m = w_0; w_0 = w_p;
            e_m = e_0; e_0 = e_p;
        }
    }
}

}  // namespace hw
