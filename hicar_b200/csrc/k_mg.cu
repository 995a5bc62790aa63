// k_mg.cu -- multigrid V-cycle preconditioner for the probed 15-point operator.
//
// The wind solver's operator couples each cell to a 5-point cross in x-y on
// the planes k-1, k, k+1, and its vertical couplings dominate (dz << dx).  The
// preconditioner is a V-cycle that respects both facts:
//   * smoother: damped z-line Jacobi, x <- x + w T^-1 (r - A x), with T the
//     tridiagonal (C, A, B) couplings of each column, solved exactly by the
//     Thomas algorithm (one thread marches one column up and down);
//   * coarsening: 2 x 2 aggregation in x-y, z kept.  The Galerkin coarse
//     operator R A P (P piecewise constant, R = P^T) of a cross stencil is again
//     a cross stencil, so every level stores the same 15 coefficients;
//   * levels continue down to a single column, where the tridiagonal solve is
//     the exact coarse solve.
// Per V-cycle and level: pre-smooth from zero, residual + restriction in one
// pass, and post-smooth with the prolongated correction added on the fly.
// Internals run in FP32 (the preconditioner precision); the outer BiCGStab
// vectors it reads and writes stay FP64.  The V-cycle is a fixed linear map
// (deterministic kernels, fixed level count), so plain BiCGStab applies.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <stdlib.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "mg.h"
#include "tc05.cuh"

namespace hw {


__device__ __forceinline__ bool inside(const Dims &d, int i, int k, int j)
{
    return i >= 1 && i <= d.nx && j >= 1 && j <= d.ny && k >= 1 && k <= d.nz;
}

// Programmatic dependent launch (the small levels' kernels, launched with the
// programmatic-serialization attribute): wait until every earlier kernel of the
// stream has completed and its writes are visible (a no-op for an ordinary
// launch), then let the next kernel be launched while this one runs; the next
// kernel reads nothing before its own wait.
__device__ __forceinline__ void pdl_prologue()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}


// offsets (dk, dj, di) of the 15 coefficients A..O
__constant__ int c_off[15][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 0, 1},  {0, 0, -1},
                                 {0, 1, 0},  {0, -1, 0}, {1, 0, 1},  {1, 0, -1}, {-1, 0, 1},
                                 {-1, 0, -1}, {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}};

// ---- Galerkin coarse operator: one thread per coarse interior cell ----
__global__ void galerkin_kernel(Dims f, const float *__restrict__ cf, Dims c, float *__restrict__ cc)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1, J = blockIdx.z + 1;
    if (I > c.nx) return;
    double acc[15];
#pragma unroll
    for (int q = 0; q < 15; q++) acc[q] = 0.0;
    for (int pj = 0; pj < 2; pj++)
        for (int pi = 0; pi < 2; pi++) {
            int i = 2 * I - 1 + pi, j = 2 * J - 1 + pj;
            if (i > f.nx || j > f.ny) continue;
            long long o = kidx(f, i, k, j);
#pragma unroll
            for (int q = 0; q < 15; q++) {
                int dk = c_off[q][0], dj = c_off[q][1], di = c_off[q][2];
                if (!inside(f, i + di, k + dk, j + dj)) continue; // couplings to boundary rows multiply zeros
                int Ip = (i + di + 1) >> 1, Jp = (j + dj + 1) >> 1;
                int cdi = Ip - I, cdj = Jp - J;
                // coarse slot with offset (dk, cdj, cdi)
                int slot;
                if (cdj == 0 && cdi == 0) slot = dk == 0 ? CA : (dk == 1 ? CB : CC);
                else if (cdj == 0) slot = dk == 0 ? (cdi == 1 ? CD : CE) : dk == 1 ? (cdi == 1 ? CH : CI) : (cdi == 1 ? CJ : CK);
                else slot = dk == 0 ? (cdj == 1 ? CF : CG) : dk == 1 ? (cdj == 1 ? CL : CM) : (cdj == 1 ? CN : CO);
                acc[slot] += (double)cf[(long long)q * f.npad + o];
            }
        }
    long long oc = kidx(c, I, k, J);
#pragma unroll
    for (int q = 0; q < 15; q++) cc[(long long)q * c.npad + oc] = (float)acc[q];
}

// ---- Thomas factors of each column's tridiagonal (C, A, B), couplings to the
// ghost planes dropped: minv_k = 1/(A_k - C_k cp_{k-1}), cp_k = B_k minv_k ----
__device__ __forceinline__ double fac_operand(float v, int bf16)
{
    return bf16 ? (double)__bfloat162float(__float2bfloat16_rn(v)) : (double)v;
}

// bf16 != 0: the factors of the BF16-rounded tridiagonal (the smoother stores its coefficients in BF16)
__global__ void factor_kernel(Dims d, const float *__restrict__ coef, float *__restrict__ cp, float *__restrict__ minv,
                              int bf16)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx) return;
    double cprev = 0.0;
    for (int k = 1; k <= d.nz; k++) {
        long long o = kidx(d, i, k, j);
        double a = k > 1 ? fac_operand(coef[(long long)CC * d.npad + o], bf16) : 0.0;
        double b = fac_operand(coef[(long long)CA * d.npad + o], bf16);
        double c = k < d.nz ? fac_operand(coef[(long long)CB * d.npad + o], bf16) : 0.0;
        double den = b - a * cprev;
        if (fabs(den) < 1e-30) den = copysign(1e-30, den);
        double m = 1.0 / den;
        minv[o] = (float)m;
        cprev = c * m;
        cp[o] = (float)cprev;
    }
}

// ---------------------------------------------------------------------------
// Column tiles.  A CTA owns TX x TY columns of a level and all nz levels.
// Phase 1 evaluates every (column, k) residual in parallel into shared memory
// (with the column's tridiagonal factors); phase 2 runs the Thomas recurrences
// in FP32, one thread per column, out of shared memory; phase 3 writes in
// parallel.  The serial part touches no global memory.
// ---------------------------------------------------------------------------

// Thomas recurrences of one column held in shared memory ([k][c] layout, stride tc):
// res <- T^-1 res, with T = tridiag(C, 1/m-form factors) and couplings to the ghost planes dropped.
// The operands of THOMAS_U levels are read ahead into registers, so that only
// the multiply-add chain is serial (the same operations in the same order as
// a level-by-level loop).
constexpr int THOMAS_U = 8;

__device__ __forceinline__ void thomas_column(float *s_res, const float *s_c, const float *s_m, const float *s_cp,
                                              int c, int tc, int nz)
{
    float dprev = 0.0f;
    int k = 0;
    for (; k + THOMAS_U <= nz; k += THOMAS_U) {
        float rv[THOMAS_U], cv[THOMAS_U], mv[THOMAS_U];
#pragma unroll
        for (int u = 0; u < THOMAS_U; u++) {
            int t = (k + u) * tc + c;
            rv[u] = s_res[t]; cv[u] = s_c[t]; mv[u] = s_m[t];
        }
#pragma unroll
        for (int u = 0; u < THOMAS_U; u++) {
            dprev = (rv[u] - cv[u] * dprev) * mv[u];
            s_res[(k + u) * tc + c] = dprev;
        }
    }
    for (; k < nz; k++) {
        int t = k * tc + c;
        dprev = (s_res[t] - s_c[t] * dprev) * s_m[t];
        s_res[t] = dprev;
    }
    float y = 0.0f;
    k = nz - 1;
    for (; k + 1 >= THOMAS_U; k -= THOMAS_U) {
        float rv[THOMAS_U], pv[THOMAS_U];
#pragma unroll
        for (int u = 0; u < THOMAS_U; u++) {
            int t = (k - u) * tc + c;
            rv[u] = s_res[t]; pv[u] = s_cp[t];
        }
#pragma unroll
        for (int u = 0; u < THOMAS_U; u++) {
            y = rv[u] - pv[u] * y;
            s_res[(k - u) * tc + c] = y;
        }
    }
    for (; k >= 0; k--) {
        int t = k * tc + c;
        y = s_res[t] - s_cp[t] * y;
        s_res[t] = y;
    }
}

constexpr int MG_THREADS = 256;
constexpr int MG_BATCH = 8; // independent loads in flight per thread in the staging loops

// The 15 coefficients of a row, loaded together (independent loads in flight);
// FP32 or BF16 storage (the finest level's smoother coefficients in BF16).
__device__ __forceinline__ float coef_val(float v) { return v; }
__device__ __forceinline__ float coef_val(__nv_bfloat16 v) { return __bfloat162float(v); }

__device__ __forceinline__ void load_coefs(const float *__restrict__ coef, long long npad, long long o, float (&cv)[15])
{
#pragma unroll
    for (int q = 0; q < 15; q++) cv[q] = __ldg(coef + o + (long long)q * npad);
}
__device__ __forceinline__ void load_coefs(const __nv_bfloat16 *__restrict__ coef, long long npad, long long o,
                                           float (&cv)[15])
{
#pragma unroll
    for (int q = 0; q < 15; q++) cv[q] = __bfloat162float(__ldg(coef + o + (long long)q * npad));
}

template <int SX, int SP>
__device__ __forceinline__ double stencil_regs(const float (&cv)[15], const float *xs)
{
    double y = 0.0;
#pragma unroll
    for (int q = 0; q < 15; q++) y += (double)cv[q] * (double)xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]];
    return y;
}

// The post-smoothers' residual r - A x2 of one cell (post_kernel, the
// tensor-copy kernels and the fused coarse cycle's post steps, which must agree
// bit for bit).  HICARW_MG_POST_F32 = 1 (the default): FP32 products and sums in
// the fixed term order (fmaf), one rounding of the difference; 0: exact
// products summed in FP64 (the restriction has its own switch,
// HICARW_MG_RESTRICT_F32).
// Measured at 1024x1024x64 with the benchmark's cycle: the same 10 iterations,
// the level-0 post-smoother 1.59 -> 1.41 ms per launch.
#ifndef HICARW_MG_POST_F32
#define HICARW_MG_POST_F32 1
#endif
template <int SX, int SP>
__device__ __forceinline__ float post_residual(double rv, const float (&cv)[15], const float *xs)
{
#if HICARW_MG_POST_F32
    float y = 0.0f;
#pragma unroll
    for (int q = 0; q < 15; q++) y = fmaf(cv[q], xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]], y);
    return (float)(rv - (double)y);
#else
    return (float)(rv - stencil_regs<SX, SP>(cv, xs));
#endif
}

// The restriction's fine residual r - A x1 of one cell, in FP64 for the sum
// over the children (restrict_pre_kernel and the fused coarse cycle's
// restriction steps, which must agree bit for bit).  HICARW_MG_RESTRICT_F32 = 1
// (the default): FP32 products and sums in the fixed term order (fmaf), the
// difference in FP64; 0: exact products summed in FP64.  The FP64 form converts
// all 30 operands of a cell to FP64, whose conversion rate, not the bytes, then
// bounds the wide levels' restrictions.
#ifndef HICARW_MG_RESTRICT_F32
#define HICARW_MG_RESTRICT_F32 1
#endif
template <int SX, int SP>
__device__ __forceinline__ double restrict_residual(double rv, const float (&cv)[15], const float *xs)
{
#if HICARW_MG_RESTRICT_F32
    float y = 0.0f;
#pragma unroll
    for (int q = 0; q < 15; q++) y = fmaf(cv[q], xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]], y);
    return rv - (double)y;
#else
    return rv - stencil_regs<SX, SP>(cv, xs);
#endif
}

// Pre-smoothing from zero: out = w T^-1 r.  A CTA owns TX x TY columns, all k.
template <typename TR, int TX, int TY>
__global__ void __launch_bounds__(MG_THREADS) pre_kernel(Dims d, const float *__restrict__ coef,
                                                         const float *__restrict__ cp, const float *__restrict__ minv,
                                                         const TR *__restrict__ r, float *__restrict__ out,
                                                         float omega, const SolveState *gate)
{
    pdl_prologue();
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    constexpr int TC = TX * TY;
    extern __shared__ float sm[];
    const int nz = d.nz, n = TC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n;
    const int i0 = blockIdx.x * TX + 1, j0 = blockIdx.y * TY + 1;
    const long long cofs = (long long)CC * d.npad;
    for (int base = threadIdx.x; base < n; base += MG_THREADS * 4) {
        float vr[4], vc[4], vm[4], vp[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            int t = base + u * MG_THREADS;
            int c = t % TC, k = t / TC + 1;
            int i = i0 + c % TX, j = j0 + c / TX;
            vr[u] = vc[u] = vm[u] = vp[u] = 0.0f;
            if (t < n && i <= d.nx && j <= d.ny) {
                long long o = kidx(d, i, k, j);
                vr[u] = (float)r[o];
                vc[u] = k > 1 ? __ldg(coef + cofs + o) : 0.0f;
                vm[u] = __ldg(minv + o);
                vp[u] = __ldg(cp + o);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            int t = base + u * MG_THREADS;
            if (t < n) { s_res[t] = vr[u]; s_c[t] = vc[u]; s_m[t] = vm[u]; s_cp[t] = vp[u]; }
        }
    }
    __syncthreads();
    if (threadIdx.x < TC) {
        int c = threadIdx.x;
        if (i0 + c % TX <= d.nx && j0 + c / TX <= d.ny) thomas_column(s_res, s_c, s_m, s_cp, c, TC, nz);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += MG_THREADS) {
        int c = t % TC, k = t / TC + 1;
        int i = i0 + c % TX, j = j0 + c / TX;
        if (i > d.nx || j > d.ny) continue;
        out[kidx(d, i, k, j)] = omega * s_res[t];
    }
}

// Stage fine-level x (optionally + P xc) of an (SX x SY) column window whose
// corner is (ia, ja), all k including the ghost planes, zero outside the interior.
template <int SX, int SY>
__device__ __forceinline__ void stage_window(const Dims &d, const float *__restrict__ x1, const Dims &dc,
                                             const float *__restrict__ xc, int ia, int ja, float *s_x,
                                             float cs = 1.0f)
{
    constexpr int SP = SX * SY;
    const int nst = SP * (d.nz + 2);
    for (int base = threadIdx.x; base < nst; base += MG_THREADS * MG_BATCH) {
        float v[MG_BATCH];
#pragma unroll
        for (int u = 0; u < MG_BATCH; u++) {
            int t = base + u * MG_THREADS;
            int lx = t % SX, ly = (t / SX) % SY, k = t / SP;
            int i = ia + lx, j = ja + ly;
            float a = 0.0f;
            if (t < nst && inside(d, i, k, j)) {
                a = __ldg(x1 + kidx(d, i, k, j));
                if (xc) a += cs * __ldg(xc + kidx(dc, (i + 1) >> 1, k, (j + 1) >> 1));
            }
            v[u] = a;
        }
#pragma unroll
        for (int u = 0; u < MG_BATCH; u++) {
            int t = base + u * MG_THREADS;
            if (t < nst) s_x[t] = v[u];
        }
    }
}

// Post-smoothing: out = x2 + w T^-1 (r - A x2) with x2 = x1 + P xc, x2 of the
// tile and its one-column ring staged in shared memory first.
constexpr int POST_CELLS = 4; // (column, level) residuals per thread in flight; 3 CTAs per SM by registers

template <typename TR, typename TO, int TX, int TY, typename CT = float>
__global__ void __launch_bounds__(MG_THREADS, 3) post_kernel(Dims d, const CT *__restrict__ coef,
                                                          const float *__restrict__ cp,
                                                          const float *__restrict__ minv, const TR *__restrict__ r,
                                                          const float *__restrict__ x1, Dims dc,
                                                          const float *__restrict__ xc, TO *__restrict__ out,
                                                          float omega, float cscale, const SolveState *gate)
{
    pdl_prologue();
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    constexpr int TC = TX * TY, SX = TX + 2, SY = TY + 2, SP = SX * SY;
    extern __shared__ float sm[];
    const int nz = d.nz, n = TC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n, *s_x = sm + 4 * n;
    const int i0 = blockIdx.x * TX + 1, j0 = blockIdx.y * TY + 1;
    stage_window<SX, SY>(d, x1, dc, xc, i0 - 1, j0 - 1, s_x, cscale);
    __syncthreads();
    for (int base = threadIdx.x; base < n; base += MG_THREADS * POST_CELLS) {
        float res2[POST_CELLS], vc[POST_CELLS], vm[POST_CELLS], vp[POST_CELLS];
#pragma unroll
        for (int u = 0; u < POST_CELLS; u++) {
            int t = base + u * MG_THREADS;
            int c = t % TC, k = t / TC + 1;
            int lx = c % TX, ly = c / TX;
            int i = i0 + lx, j = j0 + ly;
            res2[u] = vc[u] = vm[u] = vp[u] = 0.0f;
            if (t < n && i <= d.nx && j <= d.ny) {
                long long o = kidx(d, i, k, j);
                const float *xs = s_x + k * SP + (ly + 1) * SX + (lx + 1);
                float cv[15];
                load_coefs(coef, d.npad, o, cv);
                double rv = (double)r[o];
                vm[u] = __ldg(minv + o);
                vp[u] = __ldg(cp + o);
                vc[u] = k > 1 ? cv[CC] : 0.0f;
                res2[u] = post_residual<SX, SP>(rv, cv, xs);
            }
        }
#pragma unroll
        for (int u = 0; u < POST_CELLS; u++) {
            int t = base + u * MG_THREADS;
            if (t < n) { s_res[t] = res2[u]; s_c[t] = vc[u]; s_m[t] = vm[u]; s_cp[t] = vp[u]; }
        }
    }
    __syncthreads();
    if (threadIdx.x < TC) {
        int c = threadIdx.x;
        if (i0 + c % TX <= d.nx && j0 + c / TX <= d.ny) thomas_column(s_res, s_c, s_m, s_cp, c, TC, nz);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += MG_THREADS) {
        int c = t % TC, k = t / TC + 1;
        int lx = c % TX, ly = c / TX;
        int i = i0 + lx, j = j0 + ly;
        if (i > d.nx || j > d.ny) continue;
        float base = s_x[k * SP + (ly + 1) * SX + (lx + 1)];
        out[kidx(d, i, k, j)] = (TO)((double)base + (double)omega * (double)s_res[t]);
    }
}

// ---------------------------------------------------------------------------
// Post-smoothing fed by tensor copies.  The same arithmetic as post_kernel
// (bit-identical results), reorganised so that the loads need no registers:
// a persistent CTA per SM walks tiles of 32 columns (one j row) and, within a
// tile, chunks of PT_KC levels.  A producer warp streams every chunk's operands
// (15 coefficient rows, minv, cp, r, the x1 window and the coarse-correction
// window) into a PT_NS-stage shared-memory ring with cp.async.bulk.tensor; eight
// consumer warps form x2 = x1 + s P xc on the chunk's window and the residuals
// r - A x2 (one (column, level) cell per thread); warp 0 runs the forward
// Thomas recurrence of the chunk before releasing its stage, and the backward
// recurrence at the end of the tile, while the ring already fills with the
// next tile's chunks.  Every wait is bounded: on timeout the kernel sets *err,
// stops waiting and finishes its loops, so the CTA never hangs.
// ---------------------------------------------------------------------------
namespace pt {
constexpr int TX = 32;                  // columns per tile (x), one j row
constexpr int KC = 8;                   // levels per chunk: one per consumer warp
constexpr int NS = 3;                   // ring stages (two CTAs per SM)
constexpr int CW = 32 * KC;             // consumer threads
constexpr int THREADS = CW + 32;        // + the producer warp
constexpr int WX = TX + 2;              // x2 window row: i0-1 .. i0+TX
constexpr int WK = KC + 2;              // window levels: k0-1 .. k0+KC
constexpr int X1W = TX + 8;             // staged x1 row: i0-4 .. i0+TX+3 (16-byte aligned start)
constexpr int XCW = 24;                 // staged coarse row: I0-3 .. I0+20, I0 = i0 >> 1
template <typename CT> constexpr int b_coef() { return 15 * KC * TX * (int)sizeof(CT); }
constexpr int B_ROW = KC * TX * 4;      // minv / cp
constexpr int B_X1 = 3 * WK * X1W * 4;
constexpr int B_XC = 2 * WK * XCW * 4;
constexpr int up128(int b) { return (b + 127) / 128 * 128; }
// stage offsets for coefficient type CT
template <typename CT> constexpr int o_minv() { return b_coef<CT>(); }
template <typename CT> constexpr int o_cp() { return o_minv<CT>() + B_ROW; }
template <typename CT> constexpr int o_x1() { return o_cp<CT>() + B_ROW; }
template <typename CT> constexpr int o_xc() { return o_x1<CT>() + up128(B_X1); }
template <typename CT> constexpr int o_r() { return o_xc<CT>() + up128(B_XC); }
template <typename TR, typename CT> constexpr int stage_bytes() { return o_r<CT>() + up128(KC * TX * (int)sizeof(TR)); }
template <typename TR, typename CT> constexpr uint32_t tx_bytes()
{
    return b_coef<CT>() + 2 * B_ROW + B_X1 + B_XC + KC * TX * sizeof(TR);
}
static_assert(b_coef<float>() % 128 == 0 && b_coef<__nv_bfloat16>() % 128 == 0 && B_ROW % 128 == 0,
              "stage offsets must stay 128-byte aligned");

// dynamic shared memory of a launch for nz levels
template <typename TR, typename CT> size_t smem_bytes(int nz)
{
    return 128 + (size_t)NS * stage_bytes<TR, CT>() + (size_t)3 * nz * TX * 4 + (size_t)up128(3 * WK * WX * 4) +
           2 * NS * 8 + 16;
}
}  // namespace pt

template <typename TR, typename TO, typename CT = float>
__global__ void __launch_bounds__(pt::THREADS, 2)
    post_tma_kernel(const __grid_constant__ CUtensorMap tm_coef, const __grid_constant__ CUtensorMap tm_minv,
                    const __grid_constant__ CUtensorMap tm_cp, const __grid_constant__ CUtensorMap tm_r,
                    const __grid_constant__ CUtensorMap tm_x1, const __grid_constant__ CUtensorMap tm_xc, Dims d,
                    TO *__restrict__ out, float omega, float cscale, int ntx, int ntiles, const SolveState *gate,
                    int *err)
{
    using namespace pt;
    constexpr int SB = stage_bytes<TR, CT>();
    constexpr int O_COEF = 0, O_MINV = o_minv<CT>(), O_CP = o_cp<CT>(), O_X1 = o_x1<CT>(), O_XC = o_xc<CT>(),
                  O_R = o_r<CT>();
    extern __shared__ unsigned char pt_smem[];
    unsigned char *base = (unsigned char *)(((uintptr_t)pt_smem + 127) & ~(uintptr_t)127);
    const int nz = d.nz, nch = (nz + KC - 1) / KC;
    float *s_res = (float *)(base + NS * SB);
    float *s_cp = s_res + nz * TX;
    float *s_x2c = s_cp + nz * TX;
    float *s_x2w = s_x2c + nz * TX;
    uint64_t *full = (uint64_t *)((unsigned char *)s_x2w + up128(3 * WK * WX * 4));
    uint64_t *empty = full + NS;
    int *s_skip = (int *)(empty + NS);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        s_skip[0] = gate ? (*(volatile const int *)&gate->stop && !gate->profile) : 0;
        for (int q = 0; q < NS; q++) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        tc::mbar_fence_init();
    }
    __syncthreads();
    if (s_skip[0]) return; // the same value for every thread

    if (warp == KC) { // ---- producer ----
        if (lane != 0) return;
        bool ok = true;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            const int bx = tile % ntx, j = tile / ntx + 1, i0 = bx * TX + 1;
            for (int ch = 0; ch < nch; ch++, it++) {
                const int s = it % NS;
                if (it >= NS && !tc::mbar_wait(&empty[s], ((it / NS) - 1) & 1)) {
                    atomicExch(err, 1);
                    ok = false;
                    break;
                }
                unsigned char *st = base + s * SB;
                const int k0 = 1 + ch * KC, row = j * d.mz + k0;
                tc::mbar_expect_tx(&full[s], tx_bytes<TR, CT>());
                tc::tma_load_3d(st + O_COEF, &tm_coef, i0 + XO, row, 0, &full[s]);
                tc::tma_load_2d(st + O_MINV, &tm_minv, i0 + XO, row, &full[s]);
                tc::tma_load_2d(st + O_CP, &tm_cp, i0 + XO, row, &full[s]);
                tc::tma_load_3d(st + O_X1, &tm_x1, i0 + XO - 4, k0 - 1, j - 1, &full[s]);
                tc::tma_load_3d(st + O_XC, &tm_xc, (i0 >> 1) + XO - 3, k0 - 1, j >> 1, &full[s]);
                tc::tma_load_2d(st + O_R, &tm_r, i0 + XO, row, &full[s]);
            }
        }
        // no copy may still be in flight when the CTA ends: wait for the last stages issued
        for (int q = it > NS ? it - NS : 0; q < it; q++)
            if (!tc::mbar_wait(&full[q % NS], (q / NS) & 1)) atomicExch(err, 1);
        return;
    }

    // ---- consumers: warp w owns level k0 + w of each chunk, lane = column ----
    bool ok = true;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int bx = tile % ntx, j = tile / ntx + 1, i0 = bx * TX + 1;
        const int i = i0 + lane;
        const bool col = i <= d.nx;
        float dprev = 0.0f; // warp 0: carry of the forward recurrence
        for (int ch = 0; ch < nch; ch++, it++) {
            const int s = it % NS;
            const unsigned char *st = base + s * SB;
            if (ok && !tc::mbar_wait(&full[s], (it / NS) & 1)) {
                atomicExch(err, 1);
                ok = false;
            }
            const int k0 = 1 + ch * KC;
            // x2 = x1 + s P xc on the chunk's window, zero outside the interior
            const float *sx1 = (const float *)(st + O_X1), *sxc = (const float *)(st + O_XC);
            for (int e = tid; e < 3 * WK * WX; e += CW) {
                const int cc = e % WX, kw = (e / WX) % WK, jj = e / (WX * WK);
                const int ii = i0 - 1 + cc, kq = k0 - 1 + kw, jq = j - 1 + jj;
                float a = 0.0f;
                if (ii >= 1 && ii <= d.nx && jq >= 1 && jq <= d.ny && kq >= 1 && kq <= nz) {
                    a = sx1[(jj * WK + kw) * X1W + cc + 3];
                    a += cscale * sxc[((((j + jj) >> 1) - (j >> 1)) * WK + kw) * XCW + ((cc + 1) >> 1) + 3];
                }
                s_x2w[e] = a;
            }
            tc::named_sync(1, CW);
            const int k = k0 + warp;
            if (k <= nz) {
                const int t = (k - 1) * TX + lane;
                float res = 0.0f, x2c = 0.0f, cpv = 0.0f;
                if (col) {
                    const CT *sco = (const CT *)(st + O_COEF);
                    float cv[15];
#pragma unroll
                    for (int q = 0; q < 15; q++) cv[q] = coef_val(sco[(q * KC + warp) * TX + lane]);
                    const float *xs = s_x2w + (WK + warp + 1) * WX + lane + 1;
                    const double rv = (double)((const TR *)(st + O_R))[warp * TX + lane];
                    res = post_residual<WK * WX, WX>(rv, cv, xs);
                    x2c = xs[0];
                    cpv = ((const float *)(st + O_CP))[warp * TX + lane];
                }
                s_res[t] = res;
                s_cp[t] = cpv;
                s_x2c[t] = x2c;
            }
            tc::named_sync(1, CW);
            if (warp == 0) { // forward recurrence over the chunk, then release the stage
                if (col) {
                    const CT *sco = (const CT *)(st + O_COEF);
                    const float *smv = (const float *)(st + O_MINV);
                    float rv[KC], cv[KC], mv[KC];
#pragma unroll
                    for (int u = 0; u < KC; u++) {
                        const int kq = k0 + u;
                        const bool v = kq <= nz;
                        rv[u] = v ? s_res[(kq - 1) * TX + lane] : 0.0f;
                        cv[u] = v && kq > 1 ? coef_val(sco[(CC * KC + u) * TX + lane]) : 0.0f;
                        mv[u] = v ? smv[u * TX + lane] : 0.0f;
                    }
#pragma unroll
                    for (int u = 0; u < KC; u++) {
                        if (k0 + u > nz) break;
                        dprev = (rv[u] - cv[u] * dprev) * mv[u];
                        s_res[(k0 + u - 1) * TX + lane] = dprev;
                    }
                }
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&empty[s]);
            }
        }
        if (warp == 0 && col) { // backward recurrence of the tile's columns
            float y = 0.0f;
            int k = nz - 1;
            for (; k + 1 >= THOMAS_U; k -= THOMAS_U) {
                float rv[THOMAS_U], pv[THOMAS_U];
#pragma unroll
                for (int u = 0; u < THOMAS_U; u++) {
                    rv[u] = s_res[(k - u) * TX + lane];
                    pv[u] = s_cp[(k - u) * TX + lane];
                }
#pragma unroll
                for (int u = 0; u < THOMAS_U; u++) {
                    y = rv[u] - pv[u] * y;
                    s_res[(k - u) * TX + lane] = y;
                }
            }
            for (; k >= 0; k--) {
                y = s_res[k * TX + lane] - s_cp[k * TX + lane] * y;
                s_res[k * TX + lane] = y;
            }
        }
        tc::named_sync(1, CW);
        for (int t = tid; t < nz * TX; t += CW) {
            const int c = t % TX, k = t / TX + 1, ii = i0 + c;
            if (ii <= d.nx) out[kidx(d, ii, k, j)] = (TO)((double)s_x2c[t] + (double)omega * (double)s_res[t]);
        }
    }
}

// ---------------------------------------------------------------------------
// Post-smoothing fed by tensor copies, with the column recurrences moved off
// the consumers' path.  The producer warp and the stage layout are those of
// post_tma_kernel.  Eight consumer warps read each cell's 15 neighbours of x2
// = x1 + s P xc straight from the staged x1 and coarse rows (P is piecewise
// constant over the 2 x 2 aggregates, so a neighbour's coarse cell is an index
// shift; neighbours outside the interior count as zero), form the residuals,
// release the stage as soon as their reads are done, and hand each chunk's
// rows (residual, x2, cp, c, 1/m) to a recurrence warp through a ring of two
// slots.  No CTA barrier is taken per chunk.  The recurrence warp owns the
// tile's column arrays: it runs the forward recurrence chunk by chunk and, at
// the end of a tile, the backward one, writing each cell's result as soon as
// it is known; the consumers go on with the next tile meanwhile.  NX1: the
// iterate x1 is zero (the finest level without pre-smoothing), so its rows are
// neither loaded nor read.  Three stages: a fourth (measured with x1 zero at
// 1024x1024x64) made no difference once the per-chunk window and its barrier
// were gone.  Same statements per cell as post_tma_kernel, so the results are
// bit-identical.
// Every wait is bounded (on timeout: *err set, the loops run to their end
// without waiting).
// ---------------------------------------------------------------------------
namespace pt2 {
constexpr int NR = 2;                      // ring slots
constexpr int NS = 3;                      // stages
constexpr int RW = pt::KC;                 // recurrence warp
constexpr int PW = pt::KC + 1;             // producer warp
constexpr int THREADS = pt::CW + 64;
constexpr int RING_ROWS = 5;               // residual, x2, cp, c, 1/m
constexpr int B_SLOT = RING_ROWS * pt::KC * pt::TX * 4;
template <typename CT, bool NX1> constexpr int o_xc() { return pt::o_x1<CT>() + (NX1 ? 0 : pt::up128(pt::B_X1)); }
template <typename CT, bool NX1> constexpr int o_r() { return o_xc<CT, NX1>() + pt::up128(pt::B_XC); }
template <typename TR, typename CT, bool NX1> constexpr int stage_bytes()
{
    return o_r<CT, NX1>() + pt::up128(pt::KC * pt::TX * (int)sizeof(TR));
}
template <typename TR, typename CT, bool NX1> constexpr uint32_t tx_bytes()
{
    return pt::tx_bytes<TR, CT>() - (NX1 ? (uint32_t)pt::B_X1 : 0u);
}
template <typename TR, typename CT, bool NX1> size_t smem_bytes(int nz)
{
    return 128 + (size_t)NS * stage_bytes<TR, CT, NX1>() + (size_t)NR * B_SLOT + (size_t)3 * pt::TX * nz * 4 +
           2 * (NS + NR) * 8 + 16;
}
}  // namespace pt2

// Offsets (dk, dj, di) of the 15 coefficients A..O as compile-time functions
// (the table c_off, for unrolled loops that need constant indices).
__host__ __device__ constexpr int off_k(int q)
{
    return (q == 1 || q == 7 || q == 8 || q == 11 || q == 12) ? 1 : (q == 2 || q == 9 || q == 10 || q == 13 || q == 14) ? -1 : 0;
}
__host__ __device__ constexpr int off_j(int q) { return (q == 5 || q == 11 || q == 13) ? 1 : (q == 6 || q == 12 || q == 14) ? -1 : 0; }
__host__ __device__ constexpr int off_i(int q) { return (q == 3 || q == 7 || q == 9) ? 1 : (q == 4 || q == 8 || q == 10) ? -1 : 0; }
constexpr int kOffTable[15][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 0, 1},  {0, 0, -1},
                                  {0, 1, 0},  {0, -1, 0}, {1, 0, 1},  {1, 0, -1}, {-1, 0, 1},
                                  {-1, 0, -1}, {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}};
constexpr bool off_functions_match(int q = 0)
{
    return q == 15 || (off_k(q) == kOffTable[q][0] && off_j(q) == kOffTable[q][1] && off_i(q) == kOffTable[q][2] &&
                       off_functions_match(q + 1));
}
static_assert(off_functions_match(), "off_k/off_j/off_i must restate the coefficient offsets of c_off");

// post_residual with the 15 neighbour values already gathered (same terms, same order).
__device__ __forceinline__ float post_residual_vals(double rv, const float (&cv)[15], const float (&xv)[15])
{
#if HICARW_MG_POST_F32
    float y = 0.0f;
#pragma unroll
    for (int q = 0; q < 15; q++) y = fmaf(cv[q], xv[q], y);
    return (float)(rv - (double)y);
#else
    double y = 0.0;
#pragma unroll
    for (int q = 0; q < 15; q++) y += (double)cv[q] * (double)xv[q];
    return (float)(rv - y);
#endif
}

template <typename TR, typename TO, typename CT, bool NX1>
__global__ void __launch_bounds__(pt2::THREADS, 2)
    post_tma2_kernel(const __grid_constant__ CUtensorMap tm_coef, const __grid_constant__ CUtensorMap tm_minv,
                     const __grid_constant__ CUtensorMap tm_cp, const __grid_constant__ CUtensorMap tm_r,
                     const __grid_constant__ CUtensorMap tm_x1, const __grid_constant__ CUtensorMap tm_xc, Dims d,
                     TO *__restrict__ out, float omega, float cscale, int ntx, int ntiles, const SolveState *gate,
                     int *err)
{
    using namespace pt;
    constexpr int NR = pt2::NR, NS = pt2::NS;
    constexpr int SB = pt2::stage_bytes<TR, CT, NX1>();
    constexpr int O_COEF = 0, O_MINV = o_minv<CT>(), O_CP = o_cp<CT>(), O_X1 = o_x1<CT>(),
                  O_XC = pt2::o_xc<CT, NX1>(), O_R = pt2::o_r<CT, NX1>();
    constexpr int SLOT = pt2::RING_ROWS * KC * TX; // floats per ring slot
    extern __shared__ unsigned char pt_smem[];
    unsigned char *base = (unsigned char *)(((uintptr_t)pt_smem + 127) & ~(uintptr_t)127);
    const int nz = d.nz, nch = (nz + KC - 1) / KC;
    float *ring = (float *)(base + NS * SB);
    float *s_d = ring + NR * SLOT; // recurrence warp: forward results, then the column solution
    float *s_cp = s_d + nz * TX;
    float *s_x2c = s_cp + nz * TX;
    uint64_t *full = (uint64_t *)(s_x2c + nz * TX);
    uint64_t *empty = full + NS;
    uint64_t *rfull = empty + NS;
    uint64_t *rempty = rfull + NR;
    int *s_skip = (int *)(rempty + NR);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        s_skip[0] = gate ? (*(volatile const int *)&gate->stop && !gate->profile) : 0;
        for (int q = 0; q < NS; q++) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], KC); // one arrival per consumer warp
        }
        for (int q = 0; q < NR; q++) {
            tc::mbar_init(&rfull[q], KC);
            tc::mbar_init(&rempty[q], 1);
        }
        tc::mbar_fence_init();
    }
    __syncthreads();
    if (s_skip[0]) return; // the same value for every thread

    if (warp == pt2::PW) { // ---- producer ----
        if (lane != 0) return;
        constexpr uint32_t txb = pt2::tx_bytes<TR, CT, NX1>();
        bool ok = true;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            const int bx = tile % ntx, j = tile / ntx + 1, i0 = bx * TX + 1;
            for (int ch = 0; ch < nch; ch++, it++) {
                const int s = it % NS;
                if (it >= NS && !tc::mbar_wait(&empty[s], ((it / NS) - 1) & 1)) {
                    atomicExch(err, 1);
                    ok = false;
                    break;
                }
                unsigned char *st = base + s * SB;
                const int k0 = 1 + ch * KC, row = j * d.mz + k0;
                tc::mbar_expect_tx(&full[s], txb);
                tc::tma_load_3d(st + O_COEF, &tm_coef, i0 + XO, row, 0, &full[s]);
                tc::tma_load_2d(st + O_MINV, &tm_minv, i0 + XO, row, &full[s]);
                tc::tma_load_2d(st + O_CP, &tm_cp, i0 + XO, row, &full[s]);
                if (!NX1) tc::tma_load_3d(st + O_X1, &tm_x1, i0 + XO - 4, k0 - 1, j - 1, &full[s]);
                tc::tma_load_3d(st + O_XC, &tm_xc, (i0 >> 1) + XO - 3, k0 - 1, j >> 1, &full[s]);
                tc::tma_load_2d(st + O_R, &tm_r, i0 + XO, row, &full[s]);
            }
        }
        // no copy may still be in flight when the CTA ends: wait for the last stages issued
        for (int q = it > NS ? it - NS : 0; q < it; q++)
            if (!tc::mbar_wait(&full[q % NS], (q / NS) & 1)) atomicExch(err, 1);
        return;
    }

    if (warp == pt2::RW) { // ---- recurrence warp: lane = column ----
        bool ok = true;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const int bx = tile % ntx, j = tile / ntx + 1, i = bx * TX + 1 + lane;
            const bool col = i <= d.nx;
            float dprev = 0.0f;
            for (int ch = 0; ch < nch; ch++, it++) {
                const int q = it % NR;
                if (ok && !tc::mbar_wait(&rfull[q], (it / NR) & 1)) {
                    atomicExch(err, 1);
                    ok = false;
                }
                const float *rs = ring + q * SLOT;
                const int k0 = 1 + ch * KC;
                if (col) {
                    float rv[KC], xv[KC], pv[KC], cv[KC], mv[KC];
#pragma unroll
                    for (int u = 0; u < KC; u++) {
                        rv[u] = rs[(0 * KC + u) * TX + lane];
                        xv[u] = rs[(1 * KC + u) * TX + lane];
                        pv[u] = rs[(2 * KC + u) * TX + lane];
                        cv[u] = rs[(3 * KC + u) * TX + lane];
                        mv[u] = rs[(4 * KC + u) * TX + lane];
                    }
#pragma unroll
                    for (int u = 0; u < KC; u++) {
                        if (k0 + u > nz) break;
                        dprev = (rv[u] - cv[u] * dprev) * mv[u];
                        const int t = (k0 + u - 1) * TX + lane;
                        s_d[t] = dprev;
                        s_cp[t] = pv[u];
                        s_x2c[t] = xv[u];
                    }
                }
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&rempty[q]);
            }
            if (col) { // backward recurrence, each level's result written as soon as it is known
                float y = 0.0f;
                int k = nz - 1;
                for (; k + 1 >= THOMAS_U; k -= THOMAS_U) {
                    float rv[THOMAS_U], pv[THOMAS_U], xv[THOMAS_U];
#pragma unroll
                    for (int u = 0; u < THOMAS_U; u++) {
                        rv[u] = s_d[(k - u) * TX + lane];
                        pv[u] = s_cp[(k - u) * TX + lane];
                        xv[u] = s_x2c[(k - u) * TX + lane];
                    }
#pragma unroll
                    for (int u = 0; u < THOMAS_U; u++) {
                        y = rv[u] - pv[u] * y;
                        out[kidx(d, i, k - u + 1, j)] = (TO)((double)xv[u] + (double)omega * (double)y);
                    }
                }
                for (; k >= 0; k--) {
                    y = s_d[k * TX + lane] - s_cp[k * TX + lane] * y;
                    out[kidx(d, i, k + 1, j)] = (TO)((double)s_x2c[k * TX + lane] + (double)omega * (double)y);
                }
            }
        }
        return;
    }

    // ---- consumers: warp w owns level k0 + w of each chunk, lane = column ----
    bool ok = true;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int bx = tile % ntx, j = tile / ntx + 1, i0 = bx * TX + 1, i = i0 + lane;
        const bool col = i <= d.nx;
        // which x-y neighbours lie inside the interior (x2 is zero on the lateral ring)
        const bool im = i >= 2, ip = i + 1 <= d.nx, jm = j >= 2, jp = j + 1 <= d.ny;
        // staged coarse row of fine row j (row j - 1 is coarse row 0, row j + 1 coarse row 1)
        const int jc = ((j + 1) >> 1) - (j >> 1);
        for (int ch = 0; ch < nch; ch++, it++) {
            const int s = it % NS, q = it % NR;
            const unsigned char *st = base + s * SB;
            if (ok && !tc::mbar_wait(&full[s], (it / NS) & 1)) {
                atomicExch(err, 1);
                ok = false;
            }
            const int k = 1 + ch * KC + warp;
            float res = 0.0f, x2c = 0.0f, cpv = 0.0f, ccv = 0.0f, mv = 0.0f;
            if (k <= nz && col) {
                const bool km = k >= 2, kp = k + 1 <= nz;
                const float *sx1 = (const float *)(st + O_X1), *sxc = (const float *)(st + O_XC);
                const CT *sco = (const CT *)(st + O_COEF);
                float cv[15], xv[15];
#pragma unroll
                for (int qq = 0; qq < 15; qq++) cv[qq] = coef_val(sco[(qq * KC + warp) * TX + lane]);
                // x2 of the 15 neighbours: x1 row jj = dj + 1, level kw = warp + 1 + dk, column
                // cc = lane + 1 + di of the staged window (i0 - 1 .. i0 + TX), zero outside the interior
#pragma unroll
                for (int qq = 0; qq < 15; qq++) {
                    const int dk = off_k(qq), dj = off_j(qq), di = off_i(qq);
                    const bool in = (di < 0 ? im : di > 0 ? ip : true) && (dj < 0 ? jm : dj > 0 ? jp : true) &&
                                    (dk < 0 ? km : dk > 0 ? kp : true);
                    const int kw = warp + 1 + dk, cc = lane + 1 + di, cr = dj < 0 ? 0 : dj > 0 ? 1 : jc;
                    float a = 0.0f;
                    if (in) {
                        if (!NX1) a = sx1[((dj + 1) * WK + kw) * X1W + cc + 3];
                        a += cscale * sxc[(cr * WK + kw) * XCW + ((cc + 1) >> 1) + 3];
                    }
                    xv[qq] = a;
                }
                const double rv = (double)((const TR *)(st + O_R))[warp * TX + lane];
                res = post_residual_vals(rv, cv, xv);
                x2c = xv[0];
                cpv = ((const float *)(st + O_CP))[warp * TX + lane];
                mv = ((const float *)(st + O_MINV))[warp * TX + lane];
                ccv = k > 1 ? cv[CC] : 0.0f;
            }
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&empty[s]); // this warp's reads of the stage are done
            if (ok && it >= NR && !tc::mbar_wait(&rempty[q], ((it / NR) - 1) & 1)) {
                atomicExch(err, 1);
                ok = false;
            }
            float *rs = ring + q * SLOT;
            rs[(0 * KC + warp) * TX + lane] = res;
            rs[(1 * KC + warp) * TX + lane] = x2c;
            rs[(2 * KC + warp) * TX + lane] = cpv;
            rs[(3 * KC + warp) * TX + lane] = ccv;
            rs[(4 * KC + warp) * TX + lane] = mv;
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&rfull[q]);
        }
    }
}

// Restriction of level f fused with the pre-smoothing of level c = f + 1:
// r_c = R^T (r_f - A_f x1_f) for a tile of TX x TY coarse columns (fine x1 of
// the children and their ring staged in shared memory; one thread sums the four
// children of a coarse cell), then out_c = w T_c^-1 r_c (w = 1 on the
// single-column level: the exact coarse solve).
// NOX: the fine iterate is zero (no pre-smoothing on level f), so r_c = R^T r_f
// and neither the fine coefficients nor x1 are read.
template <typename TR, int TX, int TY, bool NOX>
__global__ void __launch_bounds__(MG_THREADS, 3) restrict_pre_kernel(
    Dims f, const float *__restrict__ coef_f, const TR *__restrict__ r_f, const float *__restrict__ x1_f, Dims dc,
    const float *__restrict__ coef_c, const float *__restrict__ cp_c, const float *__restrict__ minv_c,
    float *__restrict__ r_c, float *__restrict__ out_c, float omega, const SolveState *gate)
{
    pdl_prologue();
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    constexpr int TC = TX * TY, FX = 2 * TX + 2, FY = 2 * TY + 2, FP = FX * FY;
    extern __shared__ float sm[];
    const int nz = f.nz, n = TC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n, *s_x = sm + 4 * n;
    const int I0 = blockIdx.x * TX + 1, J0 = blockIdx.y * TY + 1;
    if (!NOX) stage_window<FX, FY>(f, x1_f, f, nullptr, 2 * I0 - 2, 2 * J0 - 2, s_x);
    __syncthreads();
    const long long cofs = (long long)CC * dc.npad;
    for (int t = threadIdx.x; t < n; t += MG_THREADS) {
        int c = t % TC, k = t / TC + 1;
        int lX = c % TX, lY = c / TX;
        int I = I0 + lX, J = J0 + lY;
        if (I > dc.nx || J > dc.ny) continue;
        long long oc = kidx(dc, I, k, J);
        float vc = k > 1 ? coef_c[cofs + oc] : 0.0f;
        float vm = minv_c[oc], vp = cp_c[oc];
        double acc = 0.0;
#pragma unroll
        for (int pj = 0; pj < 2; pj++) {
            // the two children of row pj: coefficients and right-hand sides loaded together
            const int j = 2 * J - 1 + pj, i0c = 2 * I - 1;
            if (j > f.ny) continue;
            const bool has1 = i0c + 1 <= f.nx;
            const long long o0 = kidx(f, i0c, k, j), o1 = o0 + 1;
            if (NOX) {
                acc += (double)r_f[o0];
                if (has1) acc += (double)r_f[o1];
                continue;
            }
            float cv0[15], cv1[15];
            load_coefs(coef_f, f.npad, o0, cv0);
            double r0 = (double)r_f[o0], r1 = 0.0;
            if (has1) {
                load_coefs(coef_f, f.npad, o1, cv1);
                r1 = (double)r_f[o1];
            }
            const float *xs0 = s_x + k * FP + (2 * lY + pj + 1) * FX + (2 * lX + 1);
            acc += restrict_residual<FX, FP>(r0, cv0, xs0);
            if (has1) acc += restrict_residual<FX, FP>(r1, cv1, xs0 + 1);
        }
        float rc = (float)acc;
        r_c[oc] = rc;
        s_res[t] = rc;
        s_c[t] = vc;
        s_m[t] = vm;
        s_cp[t] = vp;
    }
    __syncthreads();
    if (threadIdx.x < TC) {
        int c = threadIdx.x;
        if (I0 + c % TX <= dc.nx && J0 + c / TX <= dc.ny) thomas_column(s_res, s_c, s_m, s_cp, c, TC, nz);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += MG_THREADS) {
        int c = t % TC, k = t / TC + 1;
        int I = I0 + c % TX, J = J0 + c / TX;
        if (I > dc.nx || J > dc.ny) continue;
        out_c[kidx(dc, I, k, J)] = omega * s_res[t];
    }
}

// ---------------------------------------------------------------------------
// Fused coarse cycle.  Below a level of at most MG_FUSE_COLS columns the
// cycle is a chain of restriction and post-smoothing steps on tiny levels
// whose time is set by launch and memory latency (10-15 us per launch for a
// few hundred KB).  One thread-block cluster runs the whole chain instead:
// the host records the steps of coarse_cycle(l0) (levels l0 .. bottom, the
// W-cycle repeats included) into a kernel parameter, and the cluster's CTAs
// walk it, each step's column tiles spread over the CTAs, a hardware cluster
// barrier (arrive.release / wait.acquire) between steps.  Every cell's
// arithmetic is that of restrict_pre_kernel and post_kernel; only the tiling
// differs (which does not change any cell's result).  Values written inside
// the kernel are read back with ld.global.cg (L2), never through the
// read-only path.
// ---------------------------------------------------------------------------
constexpr int MG_FUSE_COLS = 256;   // first fused level: nx * ny at most this (1024x1024: level 6, 16 x 16)
constexpr int MG_FUSE_STEPS = 128;  // longest recorded chain (else the per-level launches run); 128 steps
                                    // of 232 bytes keep the kernel parameter under 32 KB
constexpr int MG_FUSE_THREADS = 512;

struct CoarseStep {
    int kind;   // 0: restriction of level f + pre-smoothing of level c; 1: post-smoothing of level f
    int tx, ty; // tile in columns: of level c (kind 0) or of level f (kind 1)
    float omega, cscale;
    Dims f, c;
    const float *coef_f, *cp_f, *minv_f, *r_f, *x1_f; // level f (x1_f: the iterate restricted / corrected)
    const float *coef_c, *cp_c, *minv_c;              // kind 0: level c
    float *r_c, *out_c;                               // kind 0: coarse right-hand side and pre-smoothed iterate
    const float *xc;                                  // kind 1: coarse correction
    float *out;                                       // kind 1: post-smoothed iterate
};

struct CoarseProg {
    int n;
    CoarseStep step[MG_FUSE_STEPS];
};
static_assert(sizeof(CoarseProg) <= 32000, "the recorded chain is passed as one kernel parameter (32 KB at most)");

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_size()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// stencil_regs with runtime window strides
__device__ __forceinline__ double stencil_regs_rt(const float (&cv)[15], const float *xs, int SX, int SP)
{
    double y = 0.0;
#pragma unroll
    for (int q = 0; q < 15; q++) y += (double)cv[q] * (double)xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]];
    return y;
}
__device__ __forceinline__ double restrict_residual_rt(double rv, const float (&cv)[15], const float *xs, int SX,
                                                       int SP)
{
#if HICARW_MG_RESTRICT_F32
    float y = 0.0f;
#pragma unroll
    for (int q = 0; q < 15; q++) y = fmaf(cv[q], xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]], y);
    return rv - (double)y;
#else
    return rv - stencil_regs_rt(cv, xs, SX, SP);
#endif
}
__device__ __forceinline__ float post_residual_rt(double rv, const float (&cv)[15], const float *xs, int SX, int SP)
{
#if HICARW_MG_POST_F32
    float y = 0.0f;
#pragma unroll
    for (int q = 0; q < 15; q++) y = fmaf(cv[q], xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]], y);
    return (float)(rv - (double)y);
#else
    return (float)(rv - stencil_regs_rt(cv, xs, SX, SP));
#endif
}

// stage_window with a runtime window shape; x1 and xc are read through L2,
// MG_BATCH elements per thread in flight
__device__ __forceinline__ void stage_window_rt(const Dims &d, const float *x1, const Dims &dc, const float *xc, int ia,
                                                int ja, int SX, int SY, float *s_x, float cs)
{
    const int SP = SX * SY, nst = SP * (d.nz + 2);
    for (int base = threadIdx.x; base < nst; base += blockDim.x * MG_BATCH) {
        float a[MG_BATCH], b[MG_BATCH];
#pragma unroll
        for (int u = 0; u < MG_BATCH; u++) {
            const int t = base + u * blockDim.x;
            const int lx = t % SX, ly = (t / SX) % SY, k = t / SP;
            const int i = ia + lx, j = ja + ly;
            a[u] = b[u] = 0.0f;
            if (t < nst && inside(d, i, k, j)) {
                a[u] = __ldcg(x1 + kidx(d, i, k, j));
                if (xc) b[u] = __ldcg(xc + kidx(dc, (i + 1) >> 1, k, (j + 1) >> 1));
            }
        }
#pragma unroll
        for (int u = 0; u < MG_BATCH; u++) {
            const int t = base + u * blockDim.x;
            if (t < nst) s_x[t] = xc ? a[u] + cs * b[u] : a[u];
        }
    }
}

// restrict_pre_kernel<float, TX, TY, false> on coarse tile (bx, by)
__device__ void fused_restrict(const CoarseStep &p, int bx, int by, float *sm)
{
    const Dims &f = p.f, &dc = p.c;
    const int TX = p.tx, TY = p.ty, TC = TX * TY, FX = 2 * TX + 2, FY = 2 * TY + 2, FP = FX * FY;
    const int nz = f.nz, n = TC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n, *s_x = sm + 4 * n;
    const int I0 = bx * TX + 1, J0 = by * TY + 1;
    stage_window_rt(f, p.x1_f, f, nullptr, 2 * I0 - 2, 2 * J0 - 2, FX, FY, s_x, 1.0f);
    __syncthreads();
    const long long cofs = (long long)CC * dc.npad;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int c = t % TC, k = t / TC + 1;
        const int lX = c % TX, lY = c / TX;
        const int I = I0 + lX, J = J0 + lY;
        if (I > dc.nx || J > dc.ny) continue;
        const long long oc = kidx(dc, I, k, J);
        const float vc = k > 1 ? __ldg(p.coef_c + cofs + oc) : 0.0f;
        const float vm = __ldg(p.minv_c + oc), vp = __ldg(p.cp_c + oc);
        double acc = 0.0;
#pragma unroll
        for (int pj = 0; pj < 2; pj++) {
            const int j = 2 * J - 1 + pj, i0c = 2 * I - 1;
            if (j > f.ny) continue;
            const bool has1 = i0c + 1 <= f.nx;
            const long long o0 = kidx(f, i0c, k, j), o1 = o0 + 1;
            float cv0[15], cv1[15];
            load_coefs(p.coef_f, f.npad, o0, cv0);
            double r0 = (double)__ldcg(p.r_f + o0), r1 = 0.0;
            if (has1) {
                load_coefs(p.coef_f, f.npad, o1, cv1);
                r1 = (double)__ldcg(p.r_f + o1);
            }
            const float *xs0 = s_x + k * FP + (2 * lY + pj + 1) * FX + (2 * lX + 1);
            acc += restrict_residual_rt(r0, cv0, xs0, FX, FP);
            if (has1) acc += restrict_residual_rt(r1, cv1, xs0 + 1, FX, FP);
        }
        const float rc = (float)acc;
        p.r_c[oc] = rc;
        s_res[t] = rc;
        s_c[t] = vc;
        s_m[t] = vm;
        s_cp[t] = vp;
    }
    __syncthreads();
    if (threadIdx.x < TC) {
        const int c = threadIdx.x;
        if (I0 + c % TX <= dc.nx && J0 + c / TX <= dc.ny) thomas_column(s_res, s_c, s_m, s_cp, c, TC, nz);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int c = t % TC, k = t / TC + 1;
        const int I = I0 + c % TX, J = J0 + c / TX;
        if (I > dc.nx || J > dc.ny) continue;
        p.out_c[kidx(dc, I, k, J)] = p.omega * s_res[t];
    }
    __syncthreads(); // the next tile reuses the shared memory
}

// post_kernel<float, float, TX, TY> on tile (bx, by) of level f
__device__ void fused_post(const CoarseStep &p, int bx, int by, float *sm)
{
    const Dims &d = p.f;
    const int TX = p.tx, TY = p.ty, TC = TX * TY, SX = TX + 2, SY = TY + 2, SP = SX * SY;
    const int nz = d.nz, n = TC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n, *s_x = sm + 4 * n;
    const int i0 = bx * TX + 1, j0 = by * TY + 1;
    stage_window_rt(d, p.x1_f, p.c, p.xc, i0 - 1, j0 - 1, SX, SY, s_x, p.cscale);
    __syncthreads();
    constexpr int FB = 2; // cells per thread whose operands are in flight together
    for (int base = threadIdx.x; base < n; base += blockDim.x * FB) {
        float cv[FB][15], rr[FB], vm[FB], vp[FB];
        bool ok[FB];
#pragma unroll
        for (int u = 0; u < FB; u++) {
            const int t = base + u * blockDim.x;
            const int c = t % TC, k = t / TC + 1;
            const int i = i0 + c % TX, j = j0 + c / TX;
            ok[u] = t < n && i <= d.nx && j <= d.ny;
            rr[u] = vm[u] = vp[u] = 0.0f;
            if (ok[u]) {
                const long long o = kidx(d, i, k, j);
                load_coefs(p.coef_f, d.npad, o, cv[u]);
                rr[u] = __ldcg(p.r_f + o);
                vm[u] = __ldg(p.minv_f + o);
                vp[u] = __ldg(p.cp_f + o);
            }
        }
#pragma unroll
        for (int u = 0; u < FB; u++) {
            const int t = base + u * blockDim.x;
            if (t >= n) continue;
            const int c = t % TC, k = t / TC + 1;
            const int lx = c % TX, ly = c / TX;
            float res2 = 0.0f, vc = 0.0f;
            if (ok[u]) {
                const float *xs = s_x + k * SP + (ly + 1) * SX + (lx + 1);
                vc = k > 1 ? cv[u][CC] : 0.0f;
                res2 = post_residual_rt((double)rr[u], cv[u], xs, SX, SP);
            }
            s_res[t] = res2;
            s_c[t] = vc;
            s_m[t] = vm[u];
            s_cp[t] = vp[u];
        }
    }
    __syncthreads();
    if (threadIdx.x < TC) {
        const int c = threadIdx.x;
        if (i0 + c % TX <= d.nx && j0 + c / TX <= d.ny) thomas_column(s_res, s_c, s_m, s_cp, c, TC, nz);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int c = t % TC, k = t / TC + 1;
        const int lx = c % TX, ly = c / TX;
        const int i = i0 + lx, j = j0 + ly;
        if (i > d.nx || j > d.ny) continue;
        const float base = s_x[k * SP + (ly + 1) * SX + (lx + 1)];
        p.out[kidx(d, i, k, j)] = (float)((double)base + (double)p.omega * (double)s_res[t]);
    }
    __syncthreads();
}

// One cluster walks the recorded chain.  The stop flag was set (or not) before
// this launch, so every CTA of the cluster takes the same branch and reaches
// the same barriers.
__global__ void __launch_bounds__(MG_FUSE_THREADS) coarse_cycle_kernel(const __grid_constant__ CoarseProg prog,
                                                                       const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    extern __shared__ float sm[];
    const int rank = (int)cluster_rank(), ncta = (int)cluster_size();
    for (int q = 0; q < prog.n; q++) {
        const CoarseStep &p = prog.step[q];
        const Dims &td = p.kind == 0 ? p.c : p.f;
        const int ntx = (td.nx + p.tx - 1) / p.tx, nty = (td.ny + p.ty - 1) / p.ty;
        for (int t = rank; t < ntx * nty; t += ncta) {
            if (p.kind == 0) fused_restrict(p, t % ntx, t / ntx, sm);
            else fused_post(p, t % ntx, t / ntx, sm);
        }
        __threadfence();
        cluster_barrier();
    }
}

// ---------------------------------------------------------------------------
static Dims level_dims(int nx, int ny, int nz, float dx)
{
    Dims d;
    d.nx = nx; d.ny = ny; d.nz = nz;
    d.mx = nx + 2; d.my = ny + 2; d.mz = nz + 2;
    d.P = ((nx + 1 + XO + 1) + 7) / 8 * 8;
    d.plane = (long long)d.P * d.mz;
    d.npad = d.plane * d.my;
    d.dx = dx;
    return d;
}

void mg_free(Mg &mg)
{
    for (int l = 0; l < mg.nlev; l++) {
        MgLevel &L = mg.lev[l];
        if (l > 0 && L.coef) cudaFree((void *)L.coef);
        if (L.cp) cudaFree(L.cp);
        if (L.minv) cudaFree(L.minv);
        if (L.r) cudaFree(L.r);
        if (L.x1) cudaFree(L.x1);
        if (L.x3) cudaFree(L.x3);
        L = MgLevel();
    }
    mg.nlev = 0;
    mg.ready = 0;
    if (mg.err) cudaFree(mg.err);
    mg.err = nullptr;
    if (mg.coef0h) cudaFree(mg.coef0h);
    mg.coef0h = nullptr;
}

static int sm_count();
static int smem_optin();
static int smem_per_sm();
static void fused_setup(Mg &mg);
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

__global__ void bf16_copy_kernel(const float *__restrict__ in, __nv_bfloat16 *__restrict__ out, size_t n)
{
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        out[q] = __float2bfloat16_rn(in[q]);
}

int mg_build(Mg &mg, const Dims &fine, const float *fine_coef, cudaStream_t s)
{
    // levels down to a single column; allocation reused when the shape is unchanged
    bool same = mg.nlev > 0 && mg.lev[0].d.nx == fine.nx && mg.lev[0].d.ny == fine.ny && mg.lev[0].d.nz == fine.nz;
    if (!same) {
        mg_free(mg);
        int nx = fine.nx, ny = fine.ny, l = 0;
        // a failed allocation releases every level allocated so far (level l included)
        auto fail = [&mg](int lev) {
            mg.nlev = lev + 1;
            mg_free(mg);
            return -1;
        };
        while (true) {
            MgLevel &L = mg.lev[l];
            L.d = l == 0 ? fine : level_dims(nx, ny, fine.nz, fine.dx);
            size_t n = (size_t)L.d.npad;
            if (l > 0) {
                if (cudaMalloc((void **)&L.coef, 15 * n * sizeof(float)) != cudaSuccess) return fail(l);
                cudaMemsetAsync((void *)L.coef, 0, 15 * n * sizeof(float), s);
                if (cudaMalloc((void **)&L.r, n * sizeof(float)) != cudaSuccess) return fail(l);
                cudaMemsetAsync(L.r, 0, n * sizeof(float), s);
                if (cudaMalloc((void **)&L.x3, n * sizeof(float)) != cudaSuccess) return fail(l);
                cudaMemsetAsync(L.x3, 0, n * sizeof(float), s);
            }
            if (cudaMalloc((void **)&L.cp, n * sizeof(float)) != cudaSuccess) return fail(l);
            if (cudaMalloc((void **)&L.minv, n * sizeof(float)) != cudaSuccess) return fail(l);
            if (cudaMalloc((void **)&L.x1, n * sizeof(float)) != cudaSuccess) return fail(l);
            cudaMemsetAsync(L.x1, 0, n * sizeof(float), s);
            l++;
            if ((nx == 1 && ny == 1) || l == MG_MAX_LEVELS) break;
            nx = (nx + 1) / 2;
            ny = (ny + 1) / 2;
        }
        mg.nlev = l;
    }
    if (!mg.err) {
        if (cudaMalloc((void **)&mg.err, sizeof(int)) != cudaSuccess) return -1;
        cudaMemsetAsync(mg.err, 0, sizeof(int), s);
    }
    if (!mg.pre0 && mg.nlev > 0) // V(0,1) on the finest level: its x1 must read as zero
        cudaMemsetAsync(mg.lev[0].x1, 0, (size_t)mg.lev[0].d.npad * sizeof(float), s);
    const char *tma = getenv("HICARW_MG_TMA");
    mg.use_tma = tma && tma[0] == '0' ? 0 : tma && tma[0] == '1' ? 1 : 2;
    sm_count(); // device queries and the encoder lookup here, never inside a stream capture
    if (mg.use_tma) {
        smem_optin();
        smem_per_sm();
        if (!tensor_map_encoder()) mg.use_tma = 0;
    }
    mg.lev[0].coef = fine_coef;
    for (int l = 0; l < mg.nlev; l++) {
        MgLevel &L = mg.lev[l];
        if (l > 0) {
            const MgLevel &F = mg.lev[l - 1];
            dim3 b(64), g((L.d.nx + 63) / 64, L.d.nz, L.d.ny);
            galerkin_kernel<<<g, b, 0, s>>>(F.d, F.coef, L.d, (float *)L.coef);
            count_launch(1);
        }
        dim3 b(64), g((L.d.nx + 63) / 64, L.d.ny);
        factor_kernel<<<g, b, 0, s>>>(L.d, L.coef, L.cp, L.minv, l == 0 && mg.bf16 && !mg.pre0);
        count_launch(1);
    }
    // the finest level's smoother coefficients in BF16 (V(0,1) cycles: its post-smoother is the only
    // kernel that reads them)
    if (mg.bf16 && !mg.pre0 && mg.nlev > 0) {
        const size_t n = 15 * (size_t)mg.lev[0].d.npad;
        if (!mg.coef0h && cudaMalloc((void **)&mg.coef0h, n * sizeof(__nv_bfloat16)) != cudaSuccess) return -1;
        bf16_copy_kernel<<<(int)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(mg.lev[0].coef, mg.coef0h, n);
        count_launch(1);
    } else if (mg.coef0h) {
        cudaFree(mg.coef0h);
        mg.coef0h = nullptr;
    }
    const cudaError_t e = cudaGetLastError();
    fused_setup(mg);
    mg.ready = 1;
    return e == cudaSuccess ? 0 : -1;
}

static const char *kLevelName[3][MG_MAX_LEVELS] = {
    {"mg_pre_l0", "mg_pre_l1", "mg_pre_l2", "mg_pre_l3", "mg_pre_l4", "mg_pre_l5", "mg_pre_l6", "mg_pre_l7",
     "mg_pre_l8", "mg_pre_l9", "mg_pre_l10", "mg_pre_l11", "mg_pre_l12", "mg_pre_l13", "mg_pre_l14", "mg_pre_l15"},
    {"mg_post_l0", "mg_post_l1", "mg_post_l2", "mg_post_l3", "mg_post_l4", "mg_post_l5", "mg_post_l6", "mg_post_l7",
     "mg_post_l8", "mg_post_l9", "mg_post_l10", "mg_post_l11", "mg_post_l12", "mg_post_l13", "mg_post_l14",
     "mg_post_l15"},
    {"mg_restrict_pre_l1", "mg_restrict_pre_l1", "mg_restrict_pre_l2", "mg_restrict_pre_l3", "mg_restrict_pre_l4",
     "mg_restrict_pre_l5", "mg_restrict_pre_l6", "mg_restrict_pre_l7", "mg_restrict_pre_l8", "mg_restrict_pre_l9",
     "mg_restrict_pre_l10", "mg_restrict_pre_l11", "mg_restrict_pre_l12", "mg_restrict_pre_l13",
     "mg_restrict_pre_l14", "mg_restrict_pre_l15"}};

// Column tiles (compile-time shapes): wide tiles on the fine levels (fewer halo
// columns), 2 x 2 tiles on coarse levels so that they still spread over many CTAs.
static bool small_level(const Dims &d, int tc) { return (long long)d.nx * d.ny < (long long)tc * 2 * 148; }

// Raise a kernel's dynamic shared-memory limit to at least smem, never lower
// it: a CUDA graph captured earlier may hold a launch of the same kernel with
// more shared memory (levels and subdomains of other sizes).
static void raise_smem(const void *kernel, size_t smem)
{
    static std::mutex mu;
    static std::vector<std::pair<const void *, size_t>> set;
    if (smem <= 48 * 1024) return;
    std::lock_guard<std::mutex> lk(mu);
    for (auto &e : set)
        if (e.first == kernel) {
            if (e.second >= smem) return;
            if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess)
                e.second = smem;
            return;
        }
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess)
        set.emplace_back(kernel, smem);
}

template <typename F>
static void set_smem(F *kernel, size_t smem)
{
    raise_smem((const void *)kernel, smem);
}

// HICARW_MG_PDL=1 in the environment launches the small levels' kernels (2 x 2
// column tiles) with programmatic stream serialization: each may be launched
// while the kernel before it runs and waits in its prologue (pdl_prologue) for
// that kernel's results.  Off by default: inside the solve's CUDA graph it
// measured no faster (1024x1024x64: 8.28 against 8.33 solves/s).  Read once.
static bool mg_pdl()
{
    static const bool on = [] {
        const char *e = getenv("HICARW_MG_PDL");
        return e && e[0] == '1';
    }();
    return on;
}

template <typename K, typename... A>
static void launch_mg(bool small, K *kernel, dim3 g, size_t smem, cudaStream_t s, A... args)
{
    if (!(small && mg_pdl())) {
        kernel<<<g, MG_THREADS, smem, s>>>(args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = g;
    cfg.blockDim = dim3(MG_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename TR, int TX, int TY>
static void pre_t(const MgLevel &L, const TR *r, float *out, float omega, const SolveState *gate, cudaStream_t s)
{
    dim3 g((L.d.nx + TX - 1) / TX, (L.d.ny + TY - 1) / TY);
    size_t smem = (size_t)4 * TX * TY * L.d.nz * sizeof(float);
    set_smem(pre_kernel<TR, TX, TY>, smem);
    launch_mg(TX == 2 && TY == 2, pre_kernel<TR, TX, TY>, g, smem, s, L.d, (const float *)L.coef,
              (const float *)L.cp, (const float *)L.minv, r, out, omega, gate);
}

template <typename TR>
static void launch_pre(const MgLevel &L, int level, const TR *r, float *out, float omega, const SolveState *gate,
                       cudaStream_t s)
{
    const double N = (double)L.d.nx * L.d.ny * L.d.nz;
    ProfScope ps_(kLevelName[0][level], (sizeof(TR) + 12.0 + 4.0) * N, s);
    if (small_level(L.d, 64)) pre_t<TR, 2, 2>(L, r, out, omega, gate, s);
    else pre_t<TR, 64, 1>(L, r, out, omega, gate, s);
    count_launch(1);
}

template <typename TR, typename TO, int TX, int TY, typename CT = float>
static void post_t(const MgLevel &L, const CT *coef, const TR *r, const MgLevel &C, TO *out, float omega,
                   float cscale, const SolveState *gate, cudaStream_t s)
{
    dim3 g((L.d.nx + TX - 1) / TX, (L.d.ny + TY - 1) / TY);
    size_t smem = ((size_t)4 * TX * TY * L.d.nz + (size_t)(TX + 2) * (TY + 2) * (L.d.nz + 2)) * sizeof(float);
    set_smem(post_kernel<TR, TO, TX, TY, CT>, smem);
    launch_mg(TX * TY <= 8, post_kernel<TR, TO, TX, TY, CT>, g, smem, s, L.d, coef, (const float *)L.cp,
              (const float *)L.minv, r, (const float *)L.x1, C.d, (const float *)C.x3, out, omega, cscale, gate);
}

static std::atomic<long long> g_tma_posts{0};
long long mg_tma_posts() { return g_tma_posts.load(); }

// Column tile of the small levels' restriction and post-smoothing kernels
// (level d: the level whose columns the tiles cover): a row of 8 columns where
// that still gives two CTAs per SM, else a row of 4.  A row of 4 or 8 columns
// reads whole 32-byte sectors of the (fine) rows; 2 x 2 tiles read half or a
// quarter of each.  Measured at 1024x1024x64 (us per launch, 2 x 2 / 4 x 1 /
// 8 x 1): restriction into 64 x 64 columns 50.7 / 36.3 / 32.8, into 32 x 32
// 19.2 / 15.7 / 16.5, into 16 x 16 15.0 / 13.1 / 15.4; post-smoothing of 64 x 64
// 29.9 / 26.4 / 22.2, of 32 x 32 13.3 / 12.8 / 13.4.  HICARW_MG_SMALL_TILE=2, 4
// or 8 in the environment fixes the tile (for measurement; read once).  The
// tile does not change any cell's arithmetic.
static int small_tile(const Dims &d)
{
    static const int forced = [] {
        const char *e = getenv("HICARW_MG_SMALL_TILE");
        return e && e[0] == '2' ? 2 : e && e[0] == '4' ? 4 : e && e[0] == '8' ? 8 : 0;
    }();
    if (forced) return forced;
    return (long long)d.nx * d.ny >= 8LL * 2 * sm_count() ? 8 : 4;
}

template <typename TR, typename TO, typename CT>
static void post_small(const MgLevel &L, const CT *coef, const TR *r, const MgLevel &C, TO *out, float omega,
                       float cscale, const SolveState *gate, cudaStream_t s)
{
    const int t = small_tile(L.d);
    if (t == 4) post_t<TR, TO, 4, 1>(L, coef, r, C, out, omega, cscale, gate, s);
    else if (t == 8) post_t<TR, TO, 8, 1>(L, coef, r, C, out, omega, cscale, gate, s);
    else post_t<TR, TO, 2, 2>(L, coef, r, C, out, omega, cscale, gate, s);
}

static int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 1;
    }
    return n;
}

static int smem_optin()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    }
    return n;
}

static int smem_per_sm()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    }
    return n;
}

// The driver's tensor-map encoder, looked up through the runtime so that the
// library does not link the driver library itself (nullptr if unavailable).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// Tiled tensor map of a row-major array (innermost dimension first, strides in
// bytes of dimensions 1..rank-1), no swizzle, zero fill out of bounds.
static bool make_map(CUtensorMap *m, CUtensorMapDataType dt, cuuint32_t rank, const void *ptr, const cuuint64_t *dims,
                     const cuuint64_t *strides, const cuuint32_t *box)
{
    if (!ptr || ((uintptr_t)ptr & 15) != 0) return false;
    for (cuuint32_t q = 0; q + 1 < rank; q++)
        if (strides[q] % 16 != 0) return false;
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return false;
    const cuuint32_t es[3] = {1, 1, 1};
    return encode(m, dt, rank, const_cast<void *>(ptr), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launch post_tma2_kernel (v2) or post_tma_kernel on a wide level; false (nothing launched) when its
// conditions do not hold: shared memory for nz levels, 16-byte aligned arrays
// and row pitches.  Box x coordinates: i0 + XO = 32 bx + 8, i0 + XO - 4 and
// (i0 >> 1) + XO - 3 = 16 bx + 4, all multiples of 4 floats (2 doubles).
template <typename TR, typename TO, typename CT = float>
static bool post_tma(const MgLevel &L, const CT *coef, const TR *r, const MgLevel &C, TO *out, float omega,
                     float cscale, const SolveState *gate, int *err, cudaStream_t s, bool v2, bool x1z)
{
    using namespace pt;
    const Dims &d = L.d, &dc = C.d;
    // the recurrence-warp kernel where two of its CTAs fit on an SM, else post_tma_kernel
    const size_t smem2 = x1z ? pt2::smem_bytes<TR, CT, true>(d.nz) : pt2::smem_bytes<TR, CT, false>(d.nz);
    if (v2 && 2 * (smem2 + 1024) > (size_t)smem_per_sm()) v2 = false;
    const size_t smem = v2 ? smem2 : smem_bytes<TR, CT>(d.nz);
    if (smem > (size_t)smem_optin() || !err || dc.mz != d.mz) return false;
    const cuuint64_t rows = (cuuint64_t)d.my * d.mz;
    const cuuint64_t dco[3] = {(cuuint64_t)d.P, rows, 15},
                     sco[2] = {(cuuint64_t)d.P * sizeof(CT), (cuuint64_t)d.npad * sizeof(CT)};
    const cuuint64_t drow[2] = {(cuuint64_t)d.P, rows}, srow[1] = {(cuuint64_t)d.P * 4},
                     srr[1] = {(cuuint64_t)d.P * sizeof(TR)};
    const cuuint64_t dx1[3] = {(cuuint64_t)d.P, (cuuint64_t)d.mz, (cuuint64_t)d.my},
                     sx1[2] = {(cuuint64_t)d.P * 4, (cuuint64_t)d.plane * 4};
    const cuuint64_t dxc[3] = {(cuuint64_t)dc.P, (cuuint64_t)dc.mz, (cuuint64_t)dc.my},
                     sxc[2] = {(cuuint64_t)dc.P * 4, (cuuint64_t)dc.plane * 4};
    const cuuint32_t bco[3] = {TX, KC, 15}, brow[2] = {TX, KC}, bx1[3] = {X1W, WK, 3}, bxc[3] = {XCW, WK, 2};
    const CUtensorMapDataType f32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const CUtensorMapDataType fr = sizeof(TR) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const CUtensorMapDataType fc = sizeof(CT) == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUtensorMap m[6];
    if (!make_map(&m[0], fc, 3, coef, dco, sco, bco) || !make_map(&m[1], f32, 2, L.minv, drow, srow, brow) ||
        !make_map(&m[2], f32, 2, L.cp, drow, srow, brow) || !make_map(&m[3], fr, 2, r, drow, srr, brow) ||
        !make_map(&m[4], f32, 3, L.x1, dx1, sx1, bx1) || !make_map(&m[5], f32, 3, C.x3, dxc, sxc, bxc))
        return false;
    const int ntx = (d.nx + TX - 1) / TX, ntiles = ntx * d.ny;
    const int grid = std::min(ntiles, 2 * sm_count());
    int *e = gate ? const_cast<int *>(&gate->err) : err;
    if (v2 && x1z) {
        raise_smem((const void *)post_tma2_kernel<TR, TO, CT, true>, smem);
        post_tma2_kernel<TR, TO, CT, true><<<grid, pt2::THREADS, smem, s>>>(m[0], m[1], m[2], m[3], m[4], m[5], d,
                                                                            out, omega, cscale, ntx, ntiles, gate, e);
    } else if (v2) {
        raise_smem((const void *)post_tma2_kernel<TR, TO, CT, false>, smem);
        post_tma2_kernel<TR, TO, CT, false><<<grid, pt2::THREADS, smem, s>>>(m[0], m[1], m[2], m[3], m[4], m[5], d,
                                                                             out, omega, cscale, ntx, ntiles, gate, e);
    } else {
        raise_smem((const void *)post_tma_kernel<TR, TO, CT>, smem);
        post_tma_kernel<TR, TO, CT><<<grid, THREADS, smem, s>>>(m[0], m[1], m[2], m[3], m[4], m[5], d, out, omega,
                                                                cscale, ntx, ntiles, gate, e);
    }
    g_tma_posts++;
    return true;
}

// coefh: the level's coefficients in BF16 (the finest level with mg_precision BF16), else nullptr;
// x1z: the level's iterate x1 is zero (the finest level without pre-smoothing);
// the recurrence-warp kernel then neither loads nor reads it.
template <typename TR, typename TO>
static void launch_post(const MgLevel &L, int level, const TR *r, const MgLevel &C, TO *out, float omega,
                        float cscale, const SolveState *gate, int use_tma, int *err, cudaStream_t s,
                        const __nv_bfloat16 *coefh = nullptr, bool x1z = false)
{
    const double N = (double)L.d.nx * L.d.ny * L.d.nz;
    const bool v2 = use_tma == 2, skip = v2 && x1z && !small_level(L.d, 32);
    ProfScope ps_(kLevelName[1][level],
                  (sizeof(TR) + sizeof(TO) + (coefh ? 30.0 : 60.0) + (skip ? 0.0 : 4.0) + 1.0 + 8.0) * N, s);
    if (coefh) {
        if (small_level(L.d, 32)) post_small<TR, TO>(L, coefh, r, C, out, omega, cscale, gate, s);
        else if (!(use_tma && post_tma<TR, TO>(L, coefh, r, C, out, omega, cscale, gate, err, s, v2, x1z)))
            post_t<TR, TO, 32, 1>(L, coefh, r, C, out, omega, cscale, gate, s);
    } else if (small_level(L.d, 32)) post_small<TR, TO>(L, L.coef, r, C, out, omega, cscale, gate, s);
    else if (!(use_tma && post_tma<TR, TO>(L, L.coef, r, C, out, omega, cscale, gate, err, s, v2, x1z)))
        post_t<TR, TO, 32, 1>(L, L.coef, r, C, out, omega, cscale, gate, s);
    count_launch(1);
}

template <typename TR, int TX, int TY, bool NOX>
static void restrict_t(const MgLevel &F, const TR *r, const MgLevel &C, float *out, float omega,
                       const SolveState *gate, cudaStream_t s)
{
    dim3 g((C.d.nx + TX - 1) / TX, (C.d.ny + TY - 1) / TY);
    size_t smem = ((size_t)4 * TX * TY * C.d.nz + (NOX ? 0 : (size_t)(2 * TX + 2) * (2 * TY + 2) * (C.d.nz + 2))) *
                  sizeof(float);
    set_smem(restrict_pre_kernel<TR, TX, TY, NOX>, smem);
    launch_mg(TX * TY <= 8, restrict_pre_kernel<TR, TX, TY, NOX>, g, smem, s, F.d, (const float *)F.coef, r,
              (const float *)F.x1, C.d, (const float *)C.coef, (const float *)C.cp, (const float *)C.minv, C.r, out,
              omega, gate);
}

// nox: level f was not pre-smoothed (its x1 is zero): restrict r_f alone.
template <typename TR>
static void launch_restrict_pre(const MgLevel &F, const TR *r, const MgLevel &C, int clevel, float *out, float omega,
                                const SolveState *gate, cudaStream_t s, bool nox = false)
{
    const double N = (double)F.d.nx * F.d.ny * F.d.nz, Nc = (double)C.d.nx * C.d.ny * C.d.nz;
    ProfScope ps_(kLevelName[2][clevel], nox ? sizeof(TR) * N + 20.0 * Nc : (60.0 + sizeof(TR) + 4.0) * N, s);
    if (small_level(C.d, 16)) {
        const int t = small_tile(C.d);
        if (t == 4) {
            if (nox) restrict_t<TR, 4, 1, true>(F, r, C, out, omega, gate, s);
            else restrict_t<TR, 4, 1, false>(F, r, C, out, omega, gate, s);
        } else if (t == 8) {
            if (nox) restrict_t<TR, 8, 1, true>(F, r, C, out, omega, gate, s);
            else restrict_t<TR, 8, 1, false>(F, r, C, out, omega, gate, s);
        } else if (nox) restrict_t<TR, 2, 2, true>(F, r, C, out, omega, gate, s);
        else restrict_t<TR, 2, 2, false>(F, r, C, out, omega, gate, s);
    } else {
        if (nox) restrict_t<TR, 16, 1, true>(F, r, C, out, omega, gate, s);
        else restrict_t<TR, 16, 1, false>(F, r, C, out, omega, gate, s);
    }
    count_launch(1);
}

// ---- fused coarse cycle: recording, tiles, launch ----
static const char *kFusedName[MG_MAX_LEVELS] = {
    "mg_coarse_l0", "mg_coarse_l1", "mg_coarse_l2",  "mg_coarse_l3",  "mg_coarse_l4",  "mg_coarse_l5",
    "mg_coarse_l6", "mg_coarse_l7", "mg_coarse_l8",  "mg_coarse_l9",  "mg_coarse_l10", "mg_coarse_l11",
    "mg_coarse_l12", "mg_coarse_l13", "mg_coarse_l14", "mg_coarse_l15"};

static size_t fused_step_smem(int kind, int tx, int ty, int nz)
{
    const size_t win = kind == 0 ? (size_t)(2 * tx + 2) * (2 * ty + 2) : (size_t)(tx + 2) * (ty + 2);
    return (4 * (size_t)tx * ty * nz + win * (nz + 2)) * sizeof(float);
}

// Tile of one step: the smallest of the candidates whose tile count fits the
// cluster (one tile per CTA), else the largest; then the largest that fits the
// shared memory.  Returns false when not even one column fits.
static bool fused_tile(int kind, const Dims &td, int nz, int cn, size_t cap, int *tx, int *ty, size_t *smem)
{
    static const int cand[7][2] = {{1, 1}, {2, 1}, {2, 2}, {4, 2}, {4, 4}, {8, 4}, {8, 8}};
    int q = 6;
    for (int c = 0; c < 7; c++)
        if ((long long)((td.nx + cand[c][0] - 1) / cand[c][0]) * ((td.ny + cand[c][1] - 1) / cand[c][1]) <= cn) {
            q = c;
            break;
        }
    for (; q >= 0; q--)
        if (fused_step_smem(kind, cand[q][0], cand[q][1], nz) <= cap) break;
    if (q < 0) return false;
    *tx = cand[q][0];
    *ty = cand[q][1];
    *smem = std::max(*smem, fused_step_smem(kind, *tx, *ty, nz));
    return true;
}

// The steps of coarse_cycle(mg, l) below, in launch order; returns the buffer
// that holds level l's result (false in *ok when the chain is too long).
static const float *record_cycle(const Mg &mg, int l, CoarseProg &prog, bool *ok)
{
    const int L = mg.nlev;
    const MgLevel &F = mg.lev[l];
    if (l == L - 1) return F.x3;
    const MgLevel &C = mg.lev[l + 1];
    const bool last = l + 1 == L - 1;
    const int reps = (mg.wmask >> l) & 1 ? 2 : 1;
    float *cur = F.x1, *other = F.x3;
    for (int rep = 0; rep < reps && *ok; rep++) {
        if (prog.n >= MG_FUSE_STEPS) { *ok = false; break; }
        CoarseStep &a = prog.step[prog.n++];
        a = CoarseStep{};
        a.kind = 0;
        a.f = F.d; a.c = C.d;
        a.coef_f = F.coef; a.r_f = F.r; a.x1_f = cur;
        a.coef_c = C.coef; a.cp_c = C.cp; a.minv_c = C.minv; a.r_c = C.r;
        a.out_c = last ? C.x3 : C.x1;
        a.omega = last ? 1.0f : mg.omega;
        const float *xc = record_cycle(mg, l + 1, prog, ok);
        if (!*ok || prog.n >= MG_FUSE_STEPS) { *ok = false; break; }
        CoarseStep &b = prog.step[prog.n++];
        b = CoarseStep{};
        b.kind = 1;
        b.f = F.d; b.c = C.d;
        b.coef_f = F.coef; b.cp_f = F.cp; b.minv_f = F.minv; b.r_f = F.r; b.x1_f = cur;
        b.xc = xc; b.out = other;
        b.omega = mg.omega; b.cscale = mg.cscale;
        std::swap(cur, other);
    }
    return cur;
}

// Largest shared memory any step of the levels from l0 down needs.
static bool fused_smem(const Mg &mg, int l0, int cn, size_t cap, size_t *smem)
{
    *smem = 0;
    for (int l = l0; l + 1 < mg.nlev; l++) {
        int tx, ty;
        if (!fused_tile(0, mg.lev[l + 1].d, mg.lev[l].d.nz, cn, cap, &tx, &ty, smem)) return false;
        if (!fused_tile(1, mg.lev[l].d, mg.lev[l].d.nz, cn, cap, &tx, &ty, smem)) return false;
    }
    return true;
}

static cudaLaunchConfig_t fused_config(int cn, size_t smem, cudaStream_t s, cudaLaunchAttribute *at)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cn);
    cfg.blockDim = dim3(MG_FUSE_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cn;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

// Decide at build time (outside any stream capture) whether and where the
// coarse part is fused (HICARW_MG_FUSE=0 in the environment: never), and the
// cluster size: 16 CTAs where the device can place such a cluster with this
// shared memory, else 8, else no fusion.  Measured at 1024x1024x64 with W on
// levels 2-4: fused from level 6 (16 x 16 columns) 8.63 solves/s against 8.56
// with one launch per level; from level 5 (32 x 32) 8.30 against 8.37; one CTA
// walking the chain from level 7 8.30.
static void fused_setup(Mg &mg)
{
    mg.fuse_level = 0;
    mg.cluster_n = 0;
    const char *e = getenv("HICARW_MG_FUSE");
    if (e && e[0] == '0') return; // one launch per level
    // HICARW_MG_FUSE_COLS: the first fused level has at most this many columns
    // (default MG_FUSE_COLS); HICARW_MG_FUSE_CTAS: the cluster size (default 16,
    // else 8; 1: one CTA walks the chain)
    const char *ec = getenv("HICARW_MG_FUSE_COLS"), *en = getenv("HICARW_MG_FUSE_CTAS");
    const long long cols = ec ? std::max(1, std::min(1024, atoi(ec))) : MG_FUSE_COLS;
    const int want = en ? atoi(en) : 0;
    int l0 = 0;
    for (int l = 2; l + 1 < mg.nlev; l++)
        if ((long long)mg.lev[l].d.nx * mg.lev[l].d.ny <= cols) {
            l0 = l;
            break;
        }
    if (!l0) return;
    if (cudaFuncSetAttribute(coarse_cycle_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    for (int cn : {16, 8, 1}) {
        if (want > 0 ? cn != want : cn == 1) continue;
        size_t smem = 0;
        if (!fused_smem(mg, l0, cn, (size_t)smem_optin(), &smem)) continue;
        raise_smem((const void *)coarse_cycle_kernel, smem);
        cudaLaunchAttribute at[1];
        cudaLaunchConfig_t cfg = fused_config(cn, smem, nullptr, at);
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, coarse_cycle_kernel, &cfg) == cudaSuccess && nclusters >= 1) {
            mg.fuse_level = l0;
            mg.cluster_n = cn;
            return;
        }
        cudaGetLastError(); // a refused size leaves no error behind
    }
}

// Enqueue coarse_cycle(mg, l) as one cluster launch; false (nothing launched)
// when the chain does not fit the recorded program or the shared memory.
static bool launch_fused(const Mg &mg, int l, const SolveState *gate, cudaStream_t s, const float **result)
{
    CoarseProg prog;
    prog.n = 0;
    bool ok = true;
    const float *res = record_cycle(mg, l, prog, &ok);
    if (!ok || prog.n == 0) return false;
    size_t smem = 0;
    double bytes = 0.0;
    for (int q = 0; q < prog.n; q++) {
        CoarseStep &p = prog.step[q];
        const Dims &td = p.kind == 0 ? p.c : p.f;
        if (!fused_tile(p.kind, td, p.f.nz, mg.cluster_n, (size_t)smem_optin(), &p.tx, &p.ty, &smem)) return false;
        const double N = (double)p.f.nx * p.f.ny * p.f.nz;
        bytes += p.kind == 0 ? (60.0 + 4.0 + 4.0) * N : (4.0 + 4.0 + 60.0 + 4.0 + 1.0 + 8.0) * N;
    }
    ProfScope ps_(kFusedName[l], bytes, s);
    raise_smem((const void *)coarse_cycle_kernel, smem);
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = fused_config(mg.cluster_n, smem, s, at);
    cudaLaunchKernelEx(&cfg, coarse_cycle_kernel, prog, gate);
    count_launch(1);
    *result = res;
    return true;
}

// Coarse part of the cycle below level l >= 1, whose right-hand side r and
// first iterate x1 (pre-smoothed from zero by the restriction kernel) are in
// place; returns the buffer that holds level l's result.  A level whose bit
// is set in mg.wmask corrects twice from the coarse grid (a W-cycle there):
// the second restriction subtracts A times the first post-smoothed iterate,
// and the two post-smoothings alternate between the level's x1 and x3 buffers.
// With no bit set the launches are those of the V-cycle: all restrictions
// top-down, then all post-smoothings bottom-up, results in x3.
static const float *coarse_cycle(const Mg &mg, int l, const SolveState *gate, cudaStream_t s)
{
    const int L = mg.nlev;
    const MgLevel &F = mg.lev[l];
    if (l == L - 1) return F.x3; // exact column solve, written by the restriction from level l - 1
    const float *fused = nullptr;
    if (mg.fuse_level > 0 && l == mg.fuse_level && launch_fused(mg, l, gate, s, &fused)) return fused;
    const MgLevel &C = mg.lev[l + 1];
    const bool last = l + 1 == L - 1;
    const int reps = (mg.wmask >> l) & 1 ? 2 : 1;
    float *cur = F.x1, *other = F.x3;
    for (int rep = 0; rep < reps; rep++) {
        MgLevel Fi = F;
        Fi.x1 = cur; // the iterate whose residual is restricted and which the post-smoother corrects
        launch_restrict_pre<float>(Fi, F.r, C, l + 1, last ? C.x3 : C.x1, last ? 1.0f : mg.omega, gate, s);
        MgLevel Cr = C;
        Cr.x3 = const_cast<float *>(coarse_cycle(mg, l + 1, gate, s));
        launch_post<float, float>(Fi, l, F.r, Cr, other, mg.omega, mg.cscale, gate, mg.use_tma, mg.err, s);
        std::swap(cur, other);
    }
    return cur;
}

// out = V-cycle(in); in/out are outer Krylov vectors of type V on the fine level.
// Launches: pre(0), restrict+pre(1..L-1) (exact solve on the last), post(L-2..0),
// with the repeated coarse corrections of the levels in mg.wmask (coarse_cycle).
// Without fine pre-smoothing (mg.pre0 == 0) pre(0) is not launched, level 1
// restricts `in` itself, and the finest post-smoother reads the zero x1.
template <typename V>
void mg_apply(const Mg &mg, const V *in, V *out, const SolveState *gate, cudaStream_t s)
{
    const int L = mg.nlev;
    const float w = mg.omega;
    if (mg.pre0) launch_pre<V>(mg.lev[0], 0, in, mg.lev[0].x1, w, gate, s);
    if (L < 2) return;
    const MgLevel &F = mg.lev[0];
    const MgLevel &C = mg.lev[1];
    const bool last = L == 2;
    launch_restrict_pre<V>(F, in, C, 1, last ? C.x3 : C.x1, last ? 1.0f : w, gate, s, !mg.pre0);
    MgLevel Cr = C;
    Cr.x3 = const_cast<float *>(coarse_cycle(mg, 1, gate, s));
    launch_post<V, V>(F, 0, in, Cr, out, w, mg.cscale, gate, mg.use_tma, mg.err, s,
                      mg.pre0 ? nullptr : mg.coef0h, !mg.pre0);
}

template void mg_apply<double>(const Mg &, const double *, double *, const SolveState *, cudaStream_t);
template void mg_apply<float>(const Mg &, const float *, float *, const SolveState *, cudaStream_t);

// ---- the bounded wait of the tensor-copy kernels, made to run out ----
// An mbarrier that expects one arrival that never comes (no copy is issued to
// it), waited on with tc::mbar_wait and a limit of limit_ns: on time-out the
// kernel records the error flag as the smoother and convolution kernels do and
// returns, leaving nothing in flight.
__global__ void wait_probe_kernel(uint64_t limit_ns, int *err)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tc::mbar_fence_init();
    }
    __syncthreads();
    const bool ok = tc::mbar_wait(&bar, 0, limit_ns);
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
}

void mg_wait_probe(int *err, uint64_t limit_ns, cudaStream_t s)
{
    wait_probe_kernel<<<1, 32, 0, s>>>(limit_ns, err);
    count_launch(1);
}

// ---- s = r - alpha v (the MG schedule applies M^-1 to s separately) ----
template <typename V>
__global__ void s_update_kernel(long long n, const V *__restrict__ r, const V *__restrict__ v, V *__restrict__ sv,
                                const SolveState *stt)
{
    if (*(volatile const int *)&stt->stop && !stt->profile) return;
    const double a = stt->alpha;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        sv[q] = (V)(1.0 * (double)r[q] + (-a) * (double)v[q]);
}

template <typename V>
void launch_s_update(const Dims &d, const V *r, const V *v, V *s, const SolveState *stt, cudaStream_t st)
{
    ProfScope ps_("s_update", (double)d.mx * d.my * d.mz * 3.0 * sizeof(V), st);
    long long b = (d.npad + 255) / 256;
    s_update_kernel<V><<<(int)(b < 148 * 16 ? b : 148 * 16), 256, 0, st>>>(d.npad, r, v, s, stt);
    count_launch(1);
}
template void launch_s_update<double>(const Dims &, const double *, const double *, double *, const SolveState *,
                                      cudaStream_t);
template void launch_s_update<float>(const Dims &, const float *, const float *, float *, const SolveState *,
                                     cudaStream_t);

}  // namespace hw
