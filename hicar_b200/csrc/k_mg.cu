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
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "mg.h"

namespace hw {


__device__ __forceinline__ bool inside(const Dims &d, int i, int k, int j)
{
    return i >= 1 && i <= d.nx && j >= 1 && j <= d.ny && k >= 1 && k <= d.nz;
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
__global__ void factor_kernel(Dims d, const float *__restrict__ coef, float *__restrict__ cp, float *__restrict__ minv)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx) return;
    double cprev = 0.0;
    for (int k = 1; k <= d.nz; k++) {
        long long o = kidx(d, i, k, j);
        double a = k > 1 ? (double)coef[(long long)CC * d.npad + o] : 0.0;
        double b = (double)coef[(long long)CA * d.npad + o];
        double c = k < d.nz ? (double)coef[(long long)CB * d.npad + o] : 0.0;
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
__device__ __forceinline__ void thomas_column(float *s_res, const float *s_c, const float *s_m, const float *s_cp,
                                              int c, int tc, int nz)
{
    float dprev = 0.0f;
    for (int k = 0; k < nz; k++) {
        int t = k * tc + c;
        float dv = (s_res[t] - s_c[t] * dprev) * s_m[t];
        s_res[t] = dv;
        dprev = dv;
    }
    float y = 0.0f;
    for (int k = nz - 1; k >= 0; k--) {
        int t = k * tc + c;
        y = s_res[t] - s_cp[t] * y;
        s_res[t] = y;
    }
}

constexpr int MG_THREADS = 256;
constexpr int MG_BATCH = 8; // independent loads in flight per thread in the staging loops

// 15-point stencil sum at padded offset o: coefficients walked with a pointer
// increment of npad through the read-only path, neighbours read from a staged
// shared-memory window.
template <int SX, int SP>
__device__ __forceinline__ double stencil_smem(const float *__restrict__ coef, long long npad, long long o,
                                               const float *xs)
{
    const float *cq = coef + o;
    double y = 0.0;
#pragma unroll
    for (int q = 0; q < 15; q++) {
        y += (double)__ldg(cq) * (double)xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]];
        cq += npad;
    }
    return y;
}

// The 15 coefficients of a row, loaded together (independent loads in flight).
__device__ __forceinline__ void load_coefs(const float *__restrict__ coef, long long npad, long long o, float (&cv)[15])
{
#pragma unroll
    for (int q = 0; q < 15; q++) cv[q] = __ldg(coef + o + (long long)q * npad);
}

template <int SX, int SP>
__device__ __forceinline__ double stencil_regs(const float (&cv)[15], const float *xs)
{
    double y = 0.0;
#pragma unroll
    for (int q = 0; q < 15; q++) y += (double)cv[q] * (double)xs[c_off[q][0] * SP + c_off[q][1] * SX + c_off[q][2]];
    return y;
}

// Pre-smoothing from zero: out = w T^-1 r.  A CTA owns TX x TY columns, all k.
template <typename TR, int TX, int TY>
__global__ void __launch_bounds__(MG_THREADS) pre_kernel(Dims d, const float *__restrict__ coef,
                                                         const float *__restrict__ cp, const float *__restrict__ minv,
                                                         const TR *__restrict__ r, float *__restrict__ out,
                                                         float omega, const SolveState *gate)
{
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
template <typename TR, typename TO, int TX, int TY>
__global__ void __launch_bounds__(MG_THREADS) post_kernel(Dims d, const float *__restrict__ coef,
                                                          const float *__restrict__ cp,
                                                          const float *__restrict__ minv, const TR *__restrict__ r,
                                                          const float *__restrict__ x1, Dims dc,
                                                          const float *__restrict__ xc, TO *__restrict__ out,
                                                          float omega, float cscale, const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    constexpr int TC = TX * TY, SX = TX + 2, SY = TY + 2, SP = SX * SY;
    extern __shared__ float sm[];
    const int nz = d.nz, n = TC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n, *s_x = sm + 4 * n;
    const int i0 = blockIdx.x * TX + 1, j0 = blockIdx.y * TY + 1;
    stage_window<SX, SY>(d, x1, dc, xc, i0 - 1, j0 - 1, s_x, cscale);
    __syncthreads();
    for (int base = threadIdx.x; base < n; base += MG_THREADS * 2) {
        float res2[2], vc[2], vm[2], vp[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
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
                res2[u] = (float)(rv - stencil_regs<SX, SP>(cv, xs));
            }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
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

// Restriction of level f fused with the pre-smoothing of level c = f + 1:
// r_c = R^T (r_f - A_f x1_f) for a tile of TX x TY coarse columns (fine x1 of
// the children and their ring staged in shared memory; one thread sums the four
// children of a coarse cell), then out_c = w T_c^-1 r_c (w = 1 on the
// single-column level: the exact coarse solve).
template <typename TR, int TX, int TY>
__global__ void __launch_bounds__(MG_THREADS, 3) restrict_pre_kernel(
    Dims f, const float *__restrict__ coef_f, const TR *__restrict__ r_f, const float *__restrict__ x1_f, Dims dc,
    const float *__restrict__ coef_c, const float *__restrict__ cp_c, const float *__restrict__ minv_c,
    float *__restrict__ r_c, float *__restrict__ out_c, float omega, const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    constexpr int TC = TX * TY, FX = 2 * TX + 2, FY = 2 * TY + 2, FP = FX * FY;
    extern __shared__ float sm[];
    const int nz = f.nz, n = TC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n, *s_x = sm + 4 * n;
    const int I0 = blockIdx.x * TX + 1, J0 = blockIdx.y * TY + 1;
    stage_window<FX, FY>(f, x1_f, f, nullptr, 2 * I0 - 2, 2 * J0 - 2, s_x);
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
            float cv0[15], cv1[15];
            load_coefs(coef_f, f.npad, o0, cv0);
            double r0 = (double)r_f[o0], r1 = 0.0;
            if (has1) {
                load_coefs(coef_f, f.npad, o1, cv1);
                r1 = (double)r_f[o1];
            }
            const float *xs0 = s_x + k * FP + (2 * lY + pj + 1) * FX + (2 * lX + 1);
            acc += r0 - stencil_regs<FX, FP>(cv0, xs0);
            if (has1) acc += r1 - stencil_regs<FX, FP>(cv1, xs0 + 1);
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
}

int mg_build(Mg &mg, const Dims &fine, const float *fine_coef, cudaStream_t s)
{
    // levels down to a single column; allocation reused when the shape is unchanged
    bool same = mg.nlev > 0 && mg.lev[0].d.nx == fine.nx && mg.lev[0].d.ny == fine.ny && mg.lev[0].d.nz == fine.nz;
    if (!same) {
        mg_free(mg);
        int nx = fine.nx, ny = fine.ny, l = 0;
        while (true) {
            MgLevel &L = mg.lev[l];
            L.d = l == 0 ? fine : level_dims(nx, ny, fine.nz, fine.dx);
            size_t n = (size_t)L.d.npad;
            if (l > 0) {
                if (cudaMalloc((void **)&L.coef, 15 * n * sizeof(float)) != cudaSuccess) return -1;
                cudaMemsetAsync((void *)L.coef, 0, 15 * n * sizeof(float), s);
                if (cudaMalloc((void **)&L.r, n * sizeof(float)) != cudaSuccess) return -1;
                cudaMemsetAsync(L.r, 0, n * sizeof(float), s);
                if (cudaMalloc((void **)&L.x3, n * sizeof(float)) != cudaSuccess) return -1;
                cudaMemsetAsync(L.x3, 0, n * sizeof(float), s);
            }
            if (cudaMalloc((void **)&L.cp, n * sizeof(float)) != cudaSuccess) return -1;
            if (cudaMalloc((void **)&L.minv, n * sizeof(float)) != cudaSuccess) return -1;
            if (cudaMalloc((void **)&L.x1, n * sizeof(float)) != cudaSuccess) return -1;
            cudaMemsetAsync(L.x1, 0, n * sizeof(float), s);
            l++;
            if ((nx == 1 && ny == 1) || l == MG_MAX_LEVELS) break;
            nx = (nx + 1) / 2;
            ny = (ny + 1) / 2;
        }
        mg.nlev = l;
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
        factor_kernel<<<g, b, 0, s>>>(L.d, L.coef, L.cp, L.minv);
        count_launch(1);
    }
    mg.ready = 1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
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

template <typename F>
static void set_smem(F *kernel, size_t smem)
{
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <typename TR, int TX, int TY>
static void pre_t(const MgLevel &L, const TR *r, float *out, float omega, const SolveState *gate, cudaStream_t s)
{
    dim3 g((L.d.nx + TX - 1) / TX, (L.d.ny + TY - 1) / TY);
    size_t smem = (size_t)4 * TX * TY * L.d.nz * sizeof(float);
    set_smem(pre_kernel<TR, TX, TY>, smem);
    pre_kernel<TR, TX, TY><<<g, MG_THREADS, smem, s>>>(L.d, L.coef, L.cp, L.minv, r, out, omega, gate);
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

template <typename TR, typename TO, int TX, int TY>
static void post_t(const MgLevel &L, const TR *r, const MgLevel &C, TO *out, float omega, float cscale,
                   const SolveState *gate, cudaStream_t s)
{
    dim3 g((L.d.nx + TX - 1) / TX, (L.d.ny + TY - 1) / TY);
    size_t smem = ((size_t)4 * TX * TY * L.d.nz + (size_t)(TX + 2) * (TY + 2) * (L.d.nz + 2)) * sizeof(float);
    set_smem(post_kernel<TR, TO, TX, TY>, smem);
    post_kernel<TR, TO, TX, TY><<<g, MG_THREADS, smem, s>>>(L.d, L.coef, L.cp, L.minv, r, L.x1, C.d, C.x3, out,
                                                            omega, cscale, gate);
}

template <typename TR, typename TO>
static void launch_post(const MgLevel &L, int level, const TR *r, const MgLevel &C, TO *out, float omega,
                        float cscale, const SolveState *gate, cudaStream_t s)
{
    const double N = (double)L.d.nx * L.d.ny * L.d.nz;
    ProfScope ps_(kLevelName[1][level], (sizeof(TR) + sizeof(TO) + 60.0 + 4.0 + 1.0 + 8.0) * N, s);
    if (small_level(L.d, 32)) post_t<TR, TO, 2, 2>(L, r, C, out, omega, cscale, gate, s);
    else post_t<TR, TO, 32, 1>(L, r, C, out, omega, cscale, gate, s);
    count_launch(1);
}

template <typename TR, int TX, int TY>
static void restrict_t(const MgLevel &F, const TR *r, const MgLevel &C, float *out, float omega,
                       const SolveState *gate, cudaStream_t s)
{
    dim3 g((C.d.nx + TX - 1) / TX, (C.d.ny + TY - 1) / TY);
    size_t smem = ((size_t)4 * TX * TY * C.d.nz + (size_t)(2 * TX + 2) * (2 * TY + 2) * (C.d.nz + 2)) *
                  sizeof(float);
    set_smem(restrict_pre_kernel<TR, TX, TY>, smem);
    restrict_pre_kernel<TR, TX, TY><<<g, MG_THREADS, smem, s>>>(F.d, F.coef, r, F.x1, C.d, C.coef, C.cp, C.minv,
                                                                C.r, out, omega, gate);
}

template <typename TR>
static void launch_restrict_pre(const MgLevel &F, const TR *r, const MgLevel &C, int clevel, float *out, float omega,
                                const SolveState *gate, cudaStream_t s)
{
    const double N = (double)F.d.nx * F.d.ny * F.d.nz;
    ProfScope ps_(kLevelName[2][clevel], (60.0 + sizeof(TR) + 4.0) * N, s);
    if (small_level(C.d, 16)) restrict_t<TR, 2, 2>(F, r, C, out, omega, gate, s);
    else restrict_t<TR, 16, 1>(F, r, C, out, omega, gate, s);
    count_launch(1);
}

// out = V-cycle(in); in/out are outer Krylov vectors of type V on the fine level.
// Launches: pre(0), restrict+pre(1..L-1) (exact solve on the last), post(L-2..0).
template <typename V>
void mg_apply(const Mg &mg, const V *in, V *out, const SolveState *gate, cudaStream_t s)
{
    const int L = mg.nlev;
    const float w = mg.omega;
    launch_pre<V>(mg.lev[0], 0, in, mg.lev[0].x1, w, gate, s);
    for (int l = 1; l < L; l++) {
        const MgLevel &F = mg.lev[l - 1];
        MgLevel &C = const_cast<MgLevel &>(mg.lev[l]);
        const bool last = l == L - 1;
        float *o = last ? C.x3 : C.x1;
        float wl = last ? 1.0f : w;
        if (l == 1) launch_restrict_pre<V>(F, in, C, l, o, wl, gate, s);
        else launch_restrict_pre<float>(F, F.r, C, l, o, wl, gate, s);
    }
    for (int l = L - 2; l >= 0; l--) {
        const MgLevel &F = mg.lev[l];
        const MgLevel &C = mg.lev[l + 1];
        if (l == 0) launch_post<V, V>(F, 0, in, C, out, w, mg.cscale, gate, s);
        else launch_post<float, float>(F, l, F.r, C, F.x3, w, mg.cscale, gate, s);
    }
}

template void mg_apply<double>(const Mg &, const double *, double *, const SolveState *, cudaStream_t);
template void mg_apply<float>(const Mg &, const float *, float *, const SolveState *, cudaStream_t);

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
