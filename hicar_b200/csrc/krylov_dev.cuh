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


}  // namespace hw
