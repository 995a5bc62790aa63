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

// x2 at a fine cell: pre-smoothed iterate plus the prolongated coarse correction
struct X2 {
    const float *x1; // may be null (zero)
    const float *xc; // may be null (no correction)
    Dims d, dc;
    __device__ __forceinline__ double at(int i, int k, int j) const
    {
        if (!inside(d, i, k, j)) return 0.0;
        double v = x1 ? (double)x1[kidx(d, i, k, j)] : 0.0;
        if (xc) v += (double)xc[kidx(dc, (i + 1) >> 1, k, (j + 1) >> 1)];
        return v;
    }
};

__device__ __forceinline__ double stencil(const Dims &d, const float *__restrict__ coef, const X2 &x, int i, int k, int j)
{
    const long long o = kidx(d, i, k, j);
    const long long N = d.npad;
    double y = 0.0;
#pragma unroll
    for (int q = 0; q < 15; q++) {
        double xv = x.at(i + c_off[q][2], k + c_off[q][0], j + c_off[q][1]);
        y += (double)coef[(long long)q * N + o] * xv;
    }
    return y;
}

// ---- smoother: out = x2 + w T^-1 (r - A x2) ----
// (x1 == xc == null: out = w T^-1 r, the pre-smoothing step from zero)
// A CTA owns MGC consecutive columns and all nz levels.  Phase 1 evaluates the
// residuals of every (column, k) in parallel (independent loads, staged in
// shared memory with the column's tridiagonal factors); phase 2 runs the Thomas
// recurrences, one thread per column, out of shared memory; phase 3 writes the
// updated iterate in parallel.  The serial part touches no global memory.
constexpr int MGC = 32;
template <typename TR, typename TO>
__global__ void __launch_bounds__(256) smooth_kernel(Dims d, const float *__restrict__ coef,
                                                     const float *__restrict__ cp, const float *__restrict__ minv,
                                                     const TR *__restrict__ r, X2 x, TO *__restrict__ out,
                                                     float omega, const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    extern __shared__ float sm[];
    const int nz = d.nz;
    const int n = MGC * nz;
    float *s_res = sm, *s_c = sm + n, *s_m = sm + 2 * n, *s_cp = sm + 3 * n, *s_base = sm + 4 * n;
    const long long ncols = (long long)d.nx * d.ny;
    const long long col0 = (long long)blockIdx.x * MGC;
    const bool stenc = x.x1 != nullptr || x.xc != nullptr;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        int c = t % MGC, k = t / MGC + 1;
        long long col = col0 + c;
        if (col >= ncols) continue;
        int i = (int)(col % d.nx) + 1, j = (int)(col / d.nx) + 1;
        long long o = kidx(d, i, k, j);
        double res = (double)r[o];
        double base = 0.0;
        if (stenc) {
            res -= stencil(d, coef, x, i, k, j);
            base = x.at(i, k, j);
        }
        s_res[t] = (float)res;
        s_base[t] = (float)base;
        s_c[t] = k > 1 ? coef[(long long)CC * d.npad + o] : 0.0f;
        s_m[t] = minv[o];
        s_cp[t] = cp[o];
    }
    __syncthreads();
    if (threadIdx.x < MGC && col0 + threadIdx.x < ncols) {
        const int c = threadIdx.x;
        double dprev = 0.0;
        for (int k = 0; k < nz; k++) {
            int t = k * MGC + c;
            double dv = ((double)s_res[t] - (double)s_c[t] * dprev) * (double)s_m[t];
            s_res[t] = (float)dv;
            dprev = dv;
        }
        double y = 0.0;
        for (int k = nz - 1; k >= 0; k--) {
            int t = k * MGC + c;
            y = (double)s_res[t] - (double)s_cp[t] * y;
            s_res[t] = (float)y;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        int c = t % MGC, k = t / MGC + 1;
        long long col = col0 + c;
        if (col >= ncols) continue;
        int i = (int)(col % d.nx) + 1, j = (int)(col / d.nx) + 1;
        out[kidx(d, i, k, j)] = (TO)((double)s_base[t] + (double)omega * (double)s_res[t]);
    }
}

// ---- r_c(I,k,J) = sum over the 2x2 children of (r - A x1): one thread per coarse cell ----
template <typename TR>
__global__ void restrict_kernel(Dims f, const float *__restrict__ coef, const TR *__restrict__ r,
                                const float *__restrict__ x1, Dims c, float *__restrict__ rc, const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1, J = blockIdx.z + 1;
    if (I > c.nx) return;
    X2 x{x1, nullptr, f, c};
    double acc = 0.0;
    for (int pj = 0; pj < 2; pj++)
        for (int pi = 0; pi < 2; pi++) {
            int i = 2 * I - 1 + pi, j = 2 * J - 1 + pj;
            if (i > f.nx || j > f.ny) continue;
            acc += (double)r[kidx(f, i, k, j)] - stencil(f, coef, x, i, k, j);
        }
    rc[kidx(c, I, k, J)] = (float)acc;
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
    {"mg_restrict_l0", "mg_restrict_l1", "mg_restrict_l2", "mg_restrict_l3", "mg_restrict_l4", "mg_restrict_l5",
     "mg_restrict_l6", "mg_restrict_l7", "mg_restrict_l8", "mg_restrict_l9", "mg_restrict_l10", "mg_restrict_l11",
     "mg_restrict_l12", "mg_restrict_l13", "mg_restrict_l14", "mg_restrict_l15"}};

template <typename TR, typename TO>
static void launch_smooth(const MgLevel &L, int level, int post, const TR *r, X2 x, TO *out, float omega,
                          const SolveState *gate, cudaStream_t s, double bytes_per_row)
{
    ProfScope ps_(kLevelName[post][level], bytes_per_row * (double)L.d.nx * L.d.ny * L.d.nz, s);
    long long cols = (long long)L.d.nx * L.d.ny;
    size_t smem = (size_t)5 * MGC * L.d.nz * sizeof(float);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(smooth_kernel<TR, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    smooth_kernel<TR, TO><<<(unsigned)((cols + MGC - 1) / MGC), 256, smem, s>>>(L.d, L.coef, L.cp, L.minv, r, x,
                                                                                 out, omega, gate);
    count_launch(1);
}

template <typename TR>
static void launch_restrict(const MgLevel &F, int level, const TR *r, const MgLevel &C, const SolveState *gate,
                            cudaStream_t s)
{
    ProfScope ps_(kLevelName[2][level], (60.0 + sizeof(TR) + 4.0) * (double)F.d.nx * F.d.ny * F.d.nz, s);
    dim3 b(64), g((C.d.nx + 63) / 64, C.d.nz, C.d.ny);
    restrict_kernel<TR><<<g, b, 0, s>>>(F.d, F.coef, r, F.x1, C.d, C.r, gate);
    count_launch(1);
}

// out = V-cycle(in); in/out are outer Krylov vectors of type V on the fine level.
template <typename V>
void mg_apply(const Mg &mg, const V *in, V *out, const SolveState *gate, cudaStream_t s)
{
    const int L = mg.nlev;
    const float w = mg.omega;
    // down: pre-smooth from zero, then residual + restriction
    for (int l = 0; l < L - 1; l++) {
        const MgLevel &F = mg.lev[l];
        X2 none{nullptr, nullptr, F.d, F.d};
        if (l == 0) {
            launch_smooth<V, float>(F, l, 0, in, none, F.x1, w, gate, s, sizeof(V) + 12.0 + 4.0);
            launch_restrict<V>(F, l, in, mg.lev[1], gate, s);
        } else {
            launch_smooth<float, float>(F, l, 0, F.r, none, F.x1, w, gate, s, 4.0 + 12.0 + 4.0);
            launch_restrict<float>(F, l, F.r, mg.lev[l + 1], gate, s);
        }
    }
    // coarsest: one column, exact tridiagonal solve
    {
        const MgLevel &Cl = mg.lev[L - 1];
        X2 none{nullptr, nullptr, Cl.d, Cl.d};
        if (L == 1) launch_smooth<V, V>(Cl, L - 1, 0, in, none, out, 1.0f, gate, s, 2.0 * sizeof(V) + 12.0);
        else launch_smooth<float, float>(Cl, L - 1, 0, Cl.r, none, Cl.x3, 1.0f, gate, s, 20.0);
    }
    // up: post-smooth of x1 + P x3(coarser)
    for (int l = L - 2; l >= 0; l--) {
        const MgLevel &F = mg.lev[l];
        const MgLevel &Cl = mg.lev[l + 1];
        X2 x2{F.x1, Cl.x3, F.d, Cl.d};
        if (l == 0) launch_smooth<V, V>(F, l, 1, in, x2, out, w, gate, s, 2.0 * sizeof(V) + 60.0 + 4.0 + 8.0 + 1.0);
        else launch_smooth<float, float>(F, l, 1, F.r, x2, F.x3, w, gate, s, 4.0 + 60.0 + 4.0 + 8.0 + 4.0 + 1.0);
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
