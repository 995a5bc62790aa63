// k_unet.cu -- the learned preconditioner: a 3-level U-Net of tensor-core 3x3x3
// convolutions (k_conv.cu), its training step (backward pass + Adam) and its
// use as z = M(r) inside the flexible Krylov solver.  No counterpart in the
// reference.
//
// Input features per interior cell (16 channels): r / rms(r), the 14 stencil
// ratios coef_q / coef_A (q = B..O) of the probed operator, and a zero channel.
// Network (levels 0, 1, 2 = full, x-y halved, x-y quartered; z kept):
//   E0 = relu(conv_a(X0))            16 -> 16  L0
//   P1 = pool(E0)                                 L1
//   E1 = relu(conv_b(P1))            16 -> 32  L1
//   P2 = pool(E1)                                 L2
//   E2 = relu(conv_c(P2))            32 -> 32  L2
//   F2 = relu(conv_d(E2))            32 -> 32  L2
//   U1 = up(F2) + E1                              L1
//   D1 = relu(conv_e(U1))            32 -> 16  L1
//   U0 = up(D1)                                   L0
//   D0 = relu(conv_f(U0) + E0)       16 -> 16  L0
//   O  = conv_g(D0) + X0             16 -> 16  L0 (channel 0 used)
//   z  = O_0 * rms(r) / coef_A       (O_0 = r / rms gives the Jacobi step)
// pool = 2x2 x-y average (cells outside the grid count as zero), up = nearest.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include <random>
#include <vector>

#include "../../include/hicarw.h"
#include "kernels.h"
#include "krylov_dev.cuh"
#include "unet.h"

namespace hw {

enum { CV_A, CV_B, CV_C, CV_D, CV_E, CV_F, CV_G, NCONV };
static const int CSPEC[NCONV][3] = { // cin, cout, level
    {16, 16, 0}, {16, 32, 1}, {32, 32, 2}, {32, 32, 2}, {32, 16, 1}, {16, 16, 0}, {16, 16, 0}};

enum { RS_POOL = 0, RS_UP = 1, RS_POOL_BWD = 2, RS_UP_BWD = 3 };
constexpr int UNET_RED = 296; // partial-sum blocks of the reductions

}  // namespace hw

using namespace hw;

struct hicarw_unet {
    int nx[3], ny[3], nz;
    size_t woff[NCONV], boff[NCONV], nparam;
    float *P = nullptr, *Gr = nullptr, *M1 = nullptr, *M2 = nullptr;
    int adam_t = 0, nsamples = 0;
    uint4 *wf[NCONV] = {}, *wb[NCONV] = {};
    uint4 *X0 = nullptr, *E0 = nullptr, *P1 = nullptr, *E1 = nullptr, *P2 = nullptr, *E2 = nullptr, *F2 = nullptr,
          *U1 = nullptr, *D1 = nullptr, *U0 = nullptr, *D0 = nullptr;
    float *O0 = nullptr;
    float *tz = nullptr, *tr = nullptr; // interior FP32 work vectors of the residual loss
    uint4 *dO = nullptr, *dD0 = nullptr, *dU0 = nullptr, *dD1 = nullptr, *dU1 = nullptr, *dF2 = nullptr,
          *dE2 = nullptr, *dP2 = nullptr, *dE1 = nullptr, *dP1 = nullptr, *dE0 = nullptr;
    const uint4 *x_in = nullptr; // input of the last forward pass
    double *red = nullptr;       // UNET_RED partial sums
    float *scal = nullptr;       // [0] rms, [1] 1/rms, [2] loss
    int *err = nullptr;
    std::vector<void *> allocs;
};

namespace hw {

static ActDims adim(const hicarw_unet *n, int lev, int C) { return act_dims(n->nx[lev], n->ny[lev], n->nz, C); }

// ---- kernels ------------------------------------------------------------------
__device__ __forceinline__ bool ugated(const SolveState *g)
{
    return g && *(volatile const int *)&g->stop && !g->profile;
}

__device__ __forceinline__ void unpack8f(const uint4 &u, float (&f)[8])
{
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float2 t = __bfloat1622float2(h[q]);
        f[2 * q] = t.x;
        f[2 * q + 1] = t.y;
    }
}

__device__ __forceinline__ uint4 pack8f(const float (&f)[8])
{
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
    return u;
}

// pooling / upsampling and their adjoints on one channel group per thread;
// then + add, then zero where mask <= 0 (add / mask have the output's shape)
__global__ void resample_kernel(int mode, const uint4 *__restrict__ in, ActDims di, uint4 *__restrict__ out, ActDims dd,
                                const uint4 *__restrict__ add, const uint4 *__restrict__ mask, const SolveState *gate)
{
    if (ugated(gate)) return;
    const long long total = (long long)dd.nx * dd.ny * dd.nz * dd.G;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % dd.nx);
        long long r = q / dd.nx;
        const int g = (int)(r % dd.G);
        r /= dd.G;
        const int k = (int)(r % dd.nz), j = (int)(r / dd.nz);
        float v[8] = {0, 0, 0, 0, 0, 0, 0, 0}, f[8];
        if (mode == RS_POOL || mode == RS_UP_BWD) { // coarse cell from its (up to) 4 children
            const float wgt = mode == RS_POOL ? 0.25f : 1.0f;
            for (int b = 0; b < 2; b++)
                for (int a = 0; a < 2; a++) {
                    const int ii = 2 * i + a, jj = 2 * j + b;
                    if (ii < di.nx && jj < di.ny) {
                        unpack8f(in[act_unit(di, ii, k, jj, g)], f);
#pragma unroll
                        for (int e = 0; e < 8; e++) v[e] += wgt * f[e];
                    }
                }
        } else { // fine cell from its parent
            const float wgt = mode == RS_UP ? 1.0f : 0.25f;
            unpack8f(in[act_unit(di, i >> 1, k, j >> 1, g)], f);
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = wgt * f[e];
        }
        const long long o = act_unit(dd, i, k, j, g);
        if (add) {
            unpack8f(add[o], f);
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] += f[e];
        }
        if (mask) {
            unpack8f(mask[o], f);
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = f[e] > 0.0f ? v[e] : 0.0f;
        }
        out[o] = pack8f(v);
    }
}

// Vector access of the solver's FP64 vectors: cell (i, k, j) with ghost cells
// included (i in [0, nx+2)) at (j*plane + k*pitch + i + off).
struct VecView {
    long long pitch, plane;
    int off;
    __device__ __forceinline__ long long at(int i, int k, int j) const { return j * plane + k * pitch + i + off; }
};

__device__ __forceinline__ void block_partial(double acc, double *part)
{
    acc = warp_sum(acc);
    __shared__ double sh[8];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
        part[blockIdx.x] = s;
    }
}

// sum of squares of the interior of r -> per-block partials
__global__ void __launch_bounds__(256) unet_sumsq_kernel(const double *__restrict__ r, VecView vw, Dims d,
                                                         double *__restrict__ part, const SolveState *gate)
{
    if (ugated(gate)) return;
    const long long n = (long long)d.nx * d.ny * d.nz;
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % d.nx);
        const long long t = q / d.nx;
        const int k = (int)(t % d.nz), j = (int)(t / d.nz);
        const double v = r[vw.at(i + 1, k + 1, j + 1)];
        acc += v * v;
    }
    block_partial(acc, part);
}

// rms and 1/rms of r (scal[0], scal[1]) from the partials
__global__ void unet_rms_kernel(const double *__restrict__ part, int nb, long long n, float *scal,
                                const SolveState *gate)
{
    if (ugated(gate)) return;
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += part[b];
    const double rms = sqrt(s / (double)n);
    scal[0] = (float)rms;
    scal[1] = rms > 0.0 ? (float)(1.0 / rms) : 0.0f;
}

// coefficient channels 1..14 of the input features (channels 0 and 15 zero)
__global__ void feat_coef_kernel(OpCtx c, uint4 *__restrict__ X0, ActDims a)
{
    const Dims &d = c.d;
    const long long n = (long long)d.nx * d.ny * d.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % d.nx);
        const long long t = q / d.nx;
        const int k = (int)(t % d.nz), j = (int)(t / d.nz);
        const long long kk = kidx(d, i + 1, k + 1, j + 1);
        const float A = c.coef[kk];
        const float inv = A != 0.0f ? 1.0f / A : 0.0f;
        float f0[8], f1[8];
        f0[0] = 0.0f;
        for (int e = 1; e < 8; e++) f0[e] = c.coef[e * d.npad + kk] * inv;
        for (int e = 0; e < 7; e++) f1[e] = c.coef[(8 + e) * d.npad + kk] * inv;
        f1[7] = 0.0f;
        X0[act_unit(a, i, k, j, 0)] = pack8f(f0);
        X0[act_unit(a, i, k, j, 1)] = pack8f(f1);
    }
}

// channel 0 of the features: r / rms(r)
__global__ void feat_r_kernel(const double *__restrict__ r, VecView vw, Dims d, uint4 *__restrict__ X0, ActDims a,
                              const float *__restrict__ scal, const SolveState *gate)
{
    if (ugated(gate)) return;
    const float inv = scal[1];
    const long long n = (long long)d.nx * d.ny * d.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % d.nx);
        const long long t = q / d.nx;
        const int k = (int)(t % d.nz), j = (int)(t / d.nz);
        const long long u = act_unit(a, i, k, j, 0);
        uint4 w = X0[u];
        reinterpret_cast<__nv_bfloat16 *>(&w)[0] = __float2bfloat16_rn((float)r[vw.at(i + 1, k + 1, j + 1)] * inv);
        X0[u] = w;
    }
}

// z = O_0 * rms / coef_A on the interior (ghost cells untouched)
__global__ void unet_out_kernel(const float *__restrict__ O0, OpCtx c, double *__restrict__ z, VecView vw,
                                const float *__restrict__ scal, const SolveState *gate)
{
    if (ugated(gate)) return;
    const Dims &d = c.d;
    const double rms = scal[0];
    const long long n = (long long)d.nx * d.ny * d.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % d.nx);
        const long long t = q / d.nx;
        const int k = (int)(t % d.nz), j = (int)(t / d.nz);
        const float A = c.coef[kidx(d, i + 1, k + 1, j + 1)];
        z[vw.at(i + 1, k + 1, j + 1)] = A != 0.0f ? (double)O0[q] * rms / (double)A : 0.0;
    }
}

// supervised loss partials sum (O_0 - T)^2 and the output gradient 2 w (O_0 - T) / n into channel 0
__global__ void __launch_bounds__(256) unet_loss_kernel(const float *__restrict__ O0, const float *__restrict__ T, int nx,
                                                        int ny, int nz, float w, uint4 *__restrict__ dO, ActDims a,
                                                        double *__restrict__ part)
{
    const long long n = (long long)nx * ny * nz;
    const float sc = 2.0f * w / (float)n;
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx);
        const long long t = q / nx;
        const int k = (int)(t % nz), j = (int)(t / nz);
        const float e = O0[q] - T[q];
        acc += (double)e * e;
        float f[8] = {sc * e, 0, 0, 0, 0, 0, 0, 0};
        dO[act_unit(a, i, k, j, 0)] = pack8f(f);
    }
    block_partial(acc, part);
}

__global__ void unet_loss_final_kernel(const double *__restrict__ part, int nb, long long n, float w, float *scal)
{
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += part[b];
    scal[2] = (float)(w * s / (double)n);
}

// Stencil offsets (dk, dj, di) of coefficients A..O of the probed operator
// (wind_iterative.F90 spmv, probed branch).
__constant__ int c_soff[15][3] = {{0, 0, 0},   {1, 0, 0},  {-1, 0, 0}, {0, 0, 1},  {0, 0, -1},
                                  {0, 1, 0},   {0, -1, 0}, {1, 0, 1},  {1, 0, -1}, {-1, 0, 1},
                                  {-1, 0, -1}, {1, 1, 0},  {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}};

// y = A x (transpose = 0) or A^T x on the interior cells with zero values
// outside; coef is (15, ny, nz, nx), x and y are (ny, nz, nx), FP32.
__global__ void interior_stencil_kernel(const float *__restrict__ coef, const float *__restrict__ x,
                                        float *__restrict__ y, int nx, int ny, int nz, int transpose)
{
    const long long n = (long long)nx * ny * nz;
    const int sg = transpose ? -1 : 1;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx);
        const long long t = q / nx;
        const int k = (int)(t % nz), j = (int)(t / nz);
        float acc = 0.0f;
#pragma unroll
        for (int s = 0; s < 15; s++) {
            const int ii = i + sg * c_soff[s][2], kk = k + sg * c_soff[s][0], jj = j + sg * c_soff[s][1];
            if (ii < 0 || ii >= nx || kk < 0 || kk >= nz || jj < 0 || jj >= ny) continue;
            const long long p = ((long long)jj * nz + kk) * nx + ii;
            // A: row q reads x[q + off_s] with coef_s[q]; A^T: row p = q - off_s has coef_s[p] on column q
            acc += coef[s * n + (transpose ? p : q)] * x[p];
        }
        y[q] = acc;
    }
}

// z = O_0 / coef_A (the network's step for a unit-rms residual)
__global__ void unet_step_kernel(const float *__restrict__ O0, const float *__restrict__ coefA, float *__restrict__ z,
                                 long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        z[q] = coefA[q] != 0.0f ? O0[q] / coefA[q] : 0.0f;
}

// res = A z - rhat (in place over az) and the loss partials sum res^2
__global__ void __launch_bounds__(256) unet_resid_kernel(float *__restrict__ az, const float *__restrict__ rhat,
                                                         long long n, double *__restrict__ part)
{
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const float e = az[q] - rhat[q];
        az[q] = e;
        acc += (double)e * e;
    }
    block_partial(acc, part);
}

// output gradient of the residual loss: dO_0 = sc (A^T res) / coef_A into channel 0
__global__ void unet_resid_grad_kernel(const float *__restrict__ atr, const float *__restrict__ coefA, float sc,
                                       int nx, int ny, int nz, uint4 *__restrict__ dO, ActDims a)
{
    const long long n = (long long)nx * ny * nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx);
        const long long t = q / nx;
        const int k = (int)(t % nz), j = (int)(t / nz);
        float f[8] = {coefA[q] != 0.0f ? sc * atr[q] / coefA[q] : 0.0f, 0, 0, 0, 0, 0, 0, 0};
        dO[act_unit(a, i, k, j, 0)] = pack8f(f);
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters with the mean gradient
// of the accumulated samples; the gradient is cleared.
__global__ void unet_adam_kernel(float *__restrict__ P, float *__restrict__ G, float *__restrict__ M1,
                                 float *__restrict__ M2, long long n, float lr, float b1, float b2, float eps, float c1,
                                 float c2, float inv_samples)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const float g = G[q] * inv_samples;
        const float m = b1 * M1[q] + (1.0f - b1) * g;
        const float v = b2 * M2[q] + (1.0f - b2) * g * g;
        M1[q] = m;
        M2[q] = v;
        P[q] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
        G[q] = 0.0f;
    }
}

// ---- host side ------------------------------------------------------------------
static int ew_grid(long long n)
{
    long long b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

static void resample(hicarw_unet *n, int mode, const uint4 *in, int lin, uint4 *out, int lout, int C, const uint4 *add,
                     const uint4 *mask, const SolveState *gate, cudaStream_t s)
{
    const ActDims di = adim(n, lin, C), dd = adim(n, lout, C);
    const long long total = (long long)dd.nx * dd.ny * dd.nz * dd.G;
    const double rd = (mode == RS_POOL || mode == RS_UP_BWD) ? 4.0 : 0.25; // input units read per output unit
    ProfScope ps_("unet_resample", (double)total * 16.0 * (1.0 + rd + (add ? 1 : 0) + (mask ? 1 : 0)), s);
    resample_kernel<<<ew_grid(total), 256, 0, s>>>(mode, in, di, out, dd, add, mask, gate);
    count_launch(1);
}

static int conv(hicarw_unet *n, int c, bool transpose, const uint4 *in, uint4 *out, const uint4 *skip, int relu,
                const uint4 *mask, float *out0, const SolveState *gate, cudaStream_t s)
{
    const int cin = CSPEC[c][0], cout = CSPEC[c][1], lev = CSPEC[c][2];
    const int ci = transpose ? cout : cin, co = transpose ? cin : cout;
    ConvArgs a{};
    a.in = in;
    a.out = out;
    a.w = transpose ? n->wb[c] : n->wf[c];
    a.bias = transpose ? nullptr : n->P + n->boff[c];
    a.skip = skip;
    a.mask = mask;
    a.out0 = out0;
    a.din = adim(n, lev, ci);
    a.dout = adim(n, lev, co);
    a.relu = relu;
    a.err = n->err;
    a.gate = gate;
    return conv3_fwd(ci, co, a, s);
}

static int wgrad(hicarw_unet *n, int c, const uint4 *x, const uint4 *dy, cudaStream_t s)
{
    const int cin = CSPEC[c][0], cout = CSPEC[c][1], lev = CSPEC[c][2];
    WgradArgs a{};
    a.x = x;
    a.dy = dy;
    a.dw = n->Gr + n->woff[c];
    a.db = n->Gr + n->boff[c];
    a.dx = adim(n, lev, cin);
    a.ddy = adim(n, lev, cout);
    a.err = n->err;
    return conv3_wgrad(cin, cout, a, s);
}

static void pack_all(hicarw_unet *n, cudaStream_t s)
{
    for (int c = 0; c < NCONV; c++) {
        conv_pack_fwd(n->P + n->woff[c], CSPEC[c][0], CSPEC[c][1], n->wf[c], s);
        conv_pack_bwd(n->P + n->woff[c], CSPEC[c][0], CSPEC[c][1], n->wb[c], s);
    }
}

static int unet_forward(hicarw_unet *n, const uint4 *x0, const SolveState *gate, cudaStream_t s)
{
    int rc = 0;
    n->x_in = x0;
    rc |= conv(n, CV_A, false, x0, n->E0, nullptr, 1, nullptr, nullptr, gate, s);
    resample(n, RS_POOL, n->E0, 0, n->P1, 1, 16, nullptr, nullptr, gate, s);
    rc |= conv(n, CV_B, false, n->P1, n->E1, nullptr, 1, nullptr, nullptr, gate, s);
    resample(n, RS_POOL, n->E1, 1, n->P2, 2, 32, nullptr, nullptr, gate, s);
    rc |= conv(n, CV_C, false, n->P2, n->E2, nullptr, 1, nullptr, nullptr, gate, s);
    rc |= conv(n, CV_D, false, n->E2, n->F2, nullptr, 1, nullptr, nullptr, gate, s);
    resample(n, RS_UP, n->F2, 2, n->U1, 1, 32, n->E1, nullptr, gate, s);
    rc |= conv(n, CV_E, false, n->U1, n->D1, nullptr, 1, nullptr, nullptr, gate, s);
    resample(n, RS_UP, n->D1, 1, n->U0, 0, 16, nullptr, nullptr, gate, s);
    rc |= conv(n, CV_F, false, n->U0, n->D0, n->E0, 1, nullptr, nullptr, gate, s);
    rc |= conv(n, CV_G, false, n->D0, nullptr, x0, 0, nullptr, n->O0, gate, s);
    return rc;
}

// backward chain from the output gradient in dO (channel 0)
static int unet_backward_chain(hicarw_unet *n, cudaStream_t s)
{
    int rc = 0;
    rc |= wgrad(n, CV_G, n->D0, n->dO, s);
    rc |= conv(n, CV_G, true, n->dO, n->dD0, nullptr, 0, n->D0, nullptr, nullptr, s);
    rc |= wgrad(n, CV_F, n->U0, n->dD0, s);
    rc |= conv(n, CV_F, true, n->dD0, n->dU0, nullptr, 0, nullptr, nullptr, nullptr, s);
    resample(n, RS_UP_BWD, n->dU0, 0, n->dD1, 1, 16, nullptr, n->D1, nullptr, s);
    rc |= wgrad(n, CV_E, n->U1, n->dD1, s);
    rc |= conv(n, CV_E, true, n->dD1, n->dU1, nullptr, 0, nullptr, nullptr, nullptr, s);
    resample(n, RS_UP_BWD, n->dU1, 1, n->dF2, 2, 32, nullptr, n->F2, nullptr, s);
    rc |= wgrad(n, CV_D, n->E2, n->dF2, s);
    rc |= conv(n, CV_D, true, n->dF2, n->dE2, nullptr, 0, n->E2, nullptr, nullptr, s);
    rc |= wgrad(n, CV_C, n->P2, n->dE2, s);
    rc |= conv(n, CV_C, true, n->dE2, n->dP2, nullptr, 0, nullptr, nullptr, nullptr, s);
    resample(n, RS_POOL_BWD, n->dP2, 2, n->dE1, 1, 32, n->dU1, n->E1, nullptr, s);
    rc |= wgrad(n, CV_B, n->P1, n->dE1, s);
    rc |= conv(n, CV_B, true, n->dE1, n->dP1, nullptr, 0, nullptr, nullptr, nullptr, s);
    resample(n, RS_POOL_BWD, n->dP1, 1, n->dE0, 0, 16, n->dD0, n->E0, nullptr, s);
    rc |= wgrad(n, CV_A, n->x_in, n->dE0, s);
    n->nsamples++;
    return rc;
}

// supervised loss w mean((O_0 - T)^2)
static int unet_backward(hicarw_unet *n, const float *T, float w, cudaStream_t s)
{
    const long long nvox = (long long)n->nx[0] * n->ny[0] * n->nz;
    unet_loss_kernel<<<UNET_RED, 256, 0, s>>>(n->O0, T, n->nx[0], n->ny[0], n->nz, w, n->dO, adim(n, 0, 16), n->red);
    unet_loss_final_kernel<<<1, 1, 0, s>>>(n->red, UNET_RED, nvox, w, n->scal);
    count_launch(2);
    return unet_backward_chain(n, s);
}

// residual loss w mean((A z - rhat)^2) with z = O_0 / coef_A, for a unit-rms residual rhat
static int unet_backward_residual(hicarw_unet *n, const float *coef, const float *rhat, float w, cudaStream_t s)
{
    const int nx = n->nx[0], ny = n->ny[0], nz = n->nz;
    const long long nvox = (long long)nx * ny * nz;
    const int g = ew_grid(nvox);
    unet_step_kernel<<<g, 256, 0, s>>>(n->O0, coef, n->tz, nvox);
    interior_stencil_kernel<<<g, 256, 0, s>>>(coef, n->tz, n->tr, nx, ny, nz, 0);
    unet_resid_kernel<<<UNET_RED, 256, 0, s>>>(n->tr, rhat, nvox, n->red);
    unet_loss_final_kernel<<<1, 1, 0, s>>>(n->red, UNET_RED, nvox, w, n->scal);
    interior_stencil_kernel<<<g, 256, 0, s>>>(coef, n->tr, n->tz, nx, ny, nz, 1);
    unet_resid_grad_kernel<<<g, 256, 0, s>>>(n->tz, coef, 2.0f * w / (float)nvox, nx, ny, nz, n->dO, adim(n, 0, 16));
    count_launch(6);
    return unet_backward_chain(n, s);
}

static VecView padded_view(const Dims &d) { return VecView{d.P, (long long)d.P * d.mz, XO}; }
static VecView plain_view(const Dims &d) { return VecView{d.mx, (long long)d.mx * d.mz, 0}; }

static void unet_rms(hicarw_unet *n, const Dims &d, const double *r, VecView vw, const SolveState *gate, cudaStream_t s)
{
    const long long nvox = (long long)d.nx * d.ny * d.nz;
    {
        ProfScope ps_("unet_rms", (double)nvox * 8.0, s);
        unet_sumsq_kernel<<<UNET_RED, 256, 0, s>>>(r, vw, d, n->red, gate);
    }
    unet_rms_kernel<<<1, 1, 0, s>>>(n->red, UNET_RED, nvox, n->scal, gate);
    count_launch(2);
}

// z = M(r) for solver vectors in the given view
static int unet_apply(hicarw_unet *n, const OpCtx &c, const double *r, double *z, VecView vw, const SolveState *gate,
                      cudaStream_t s)
{
    const Dims &d = c.d;
    const long long nvox = (long long)d.nx * d.ny * d.nz;
    unet_rms(n, d, r, vw, gate, s);
    {
        ProfScope ps_("unet_features", (double)nvox * (8.0 + 32.0), s);
        feat_r_kernel<<<ew_grid(nvox), 256, 0, s>>>(r, vw, d, n->X0, adim(n, 0, 16), n->scal, gate);
        count_launch(1);
    }
    int rc = unet_forward(n, n->X0, gate, s);
    ProfScope ps_("unet_output", (double)nvox * 16.0, s);
    unet_out_kernel<<<ew_grid(nvox), 256, 0, s>>>(n->O0, c, z, vw, n->scal, gate);
    count_launch(1);
    return rc;
}

// ---- entry points used by the solver (capi.cu) ----
int unet_prepare_operator(hicarw_unet *n, const OpCtx &c, cudaStream_t s)
{
    if (!n || c.d.nx != n->nx[0] || c.d.ny != n->ny[0] || c.d.nz != n->nz) return -1;
    const long long nvox = (long long)c.d.nx * c.d.ny * c.d.nz;
    feat_coef_kernel<<<ew_grid(nvox), 256, 0, s>>>(c, n->X0, adim(n, 0, 16));
    count_launch(1);
    return 0;
}

int unet_precond(hicarw_unet *n, const OpCtx &c, const double *in, double *out, const SolveState *gate, cudaStream_t s)
{
    return unet_apply(n, c, in, out, padded_view(c.d), gate, s);
}

bool unet_matches(const hicarw_unet *n, const Dims &d)
{
    return n && d.nx == n->nx[0] && d.ny == n->ny[0] && d.nz == n->nz;
}

void handle_operator(const hicarw_handle *h, OpCtx *c); // capi.cu

}  // namespace hw

// ---- C entry points -------------------------------------------------------------
static int ualloc(hicarw_unet *n, void **p, size_t bytes)
{
    if (cudaMalloc(p, bytes) != cudaSuccess) return -1;
    n->allocs.push_back(*p);
    if (cudaMemset(*p, 0, bytes) != cudaSuccess) return -1;
    return 0;
}

extern "C" int hicarw_unet_destroy(hicarw_unet *n)
{
    api_entry();
    if (!n) return HICARW_ERR_ARG;
    cudaDeviceSynchronize();
    for (void *p : n->allocs) cudaFree(p);
    delete n;
    return HICARW_OK;
}

extern "C" int hicarw_unet_create(int nx, int ny, int nz, unsigned long long seed, hicarw_unet **out)
{
    api_entry();
    if (!out || nx < 1 || ny < 1 || nz < 1) return HICARW_ERR_ARG;
    hicarw_unet *n = new hicarw_unet();
    n->nx[0] = nx;
    n->ny[0] = ny;
    for (int l = 1; l < 3; l++) {
        n->nx[l] = (n->nx[l - 1] + 1) / 2;
        n->ny[l] = (n->ny[l - 1] + 1) / 2;
    }
    n->nz = nz;
    size_t off = 0;
    for (int c = 0; c < NCONV; c++) {
        n->woff[c] = off;
        off += (size_t)27 * CSPEC[c][0] * CSPEC[c][1];
        n->boff[c] = off;
        off += CSPEC[c][1];
    }
    n->nparam = off;
    bool bad = false;
    auto A = [&](void **p, size_t b) {
        if (!bad && ualloc(n, p, b)) bad = true;
    };
    A((void **)&n->P, off * 4);
    A((void **)&n->Gr, off * 4);
    A((void **)&n->M1, off * 4);
    A((void **)&n->M2, off * 4);
    for (int c = 0; c < NCONV; c++) {
        A((void **)&n->wf[c], conv_wimage_bytes(CSPEC[c][0], CSPEC[c][1]));
        A((void **)&n->wb[c], conv_wimage_bytes(CSPEC[c][0], CSPEC[c][1]));
    }
    auto T = [&](uint4 **p, int lev, int C) { A((void **)p, (size_t)act_units(adim(n, lev, C)) * 16); };
    T(&n->X0, 0, 16);
    T(&n->E0, 0, 16);
    T(&n->P1, 1, 16);
    T(&n->E1, 1, 32);
    T(&n->P2, 2, 32);
    T(&n->E2, 2, 32);
    T(&n->F2, 2, 32);
    T(&n->U1, 1, 32);
    T(&n->D1, 1, 16);
    T(&n->U0, 0, 16);
    T(&n->D0, 0, 16);
    A((void **)&n->O0, (size_t)nx * ny * nz * 4);
    A((void **)&n->red, UNET_RED * 8);
    A((void **)&n->scal, 16);
    A((void **)&n->err, 4);
    if (bad) {
        hicarw_unet_destroy(n);
        return HICARW_ERR_CUDA;
    }
    // He-normal weights (std sqrt(2 / fan_in)), zero biases; the last convolution
    // starts 10x smaller so that the initial network is close to the Jacobi step.
    std::vector<float> h(off, 0.0f);
    std::mt19937_64 rng(seed);
    for (int c = 0; c < NCONV; c++) {
        std::normal_distribution<float> nd(0.0f, sqrtf(2.0f / (27.0f * CSPEC[c][0])) * (c == CV_G ? 0.1f : 1.0f));
        for (size_t q = 0; q < (size_t)27 * CSPEC[c][0] * CSPEC[c][1]; q++) h[n->woff[c] + q] = nd(rng);
    }
    cudaMemcpy(n->P, h.data(), off * 4, cudaMemcpyHostToDevice);
    pack_all(n, 0);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        hicarw_unet_destroy(n);
        return HICARW_ERR_CUDA;
    }
    *out = n;
    return HICARW_OK;
}

static int ensure_grads(hicarw_unet *n)
{
    if (n->dO) return 0;
    auto T = [&](uint4 **p, int lev, int C) { return ualloc(n, (void **)p, (size_t)act_units(adim(n, lev, C)) * 16); };
    int bad = 0;
    bad |= T(&n->dO, 0, 16);
    bad |= T(&n->dD0, 0, 16);
    bad |= T(&n->dU0, 0, 16);
    bad |= T(&n->dD1, 1, 16);
    bad |= T(&n->dU1, 1, 32);
    bad |= T(&n->dF2, 2, 32);
    bad |= T(&n->dE2, 2, 32);
    bad |= T(&n->dP2, 2, 32);
    bad |= T(&n->dE1, 1, 32);
    bad |= T(&n->dP1, 1, 16);
    bad |= T(&n->dE0, 0, 16);
    const size_t nv = (size_t)n->nx[0] * n->ny[0] * n->nz * 4;
    bad |= ualloc(n, (void **)&n->tz, nv);
    bad |= ualloc(n, (void **)&n->tr, nv);
    return bad;
}

static int finish(hicarw_unet *n, int rc, cudaStream_t s, const char *what)
{
    int herr = 0;
    cudaMemcpyAsync(&herr, n->err, 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (rc == -2) {
        fprintf(stderr, "%s: bad convolution arguments\n", what);
        return HICARW_ERR_ARG;
    }
    if (rc != 0 || e != cudaSuccess) {
        fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError()));
        return HICARW_ERR_CUDA;
    }
    if (herr) {
        fprintf(stderr, "%s: a pipeline wait timed out\n", what);
        return HICARW_ERR_CUDA;
    }
    return HICARW_OK;
}

static cudaMemcpyKind kind_of(int mem_kind, bool to_device)
{
    if (mem_kind == HICARW_MEM_HOST) return to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    return cudaMemcpyDeviceToDevice;
}

extern "C" long long hicarw_unet_num_params(const hicarw_unet *n) {
    api_entry(); return n ? (long long)n->nparam : -1; }

extern "C" int hicarw_unet_grid(const hicarw_unet *n, int *nx, int *ny, int *nz)
{
    api_entry();
    if (!n) return HICARW_ERR_ARG;
    if (nx) *nx = n->nx[0];
    if (ny) *ny = n->ny[0];
    if (nz) *nz = n->nz;
    return HICARW_OK;
}

extern "C" int hicarw_unet_get_params(hicarw_unet *n, float *out, int mem_kind, void *stream)
{
    api_entry();
    if (!n || !out) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemcpyAsync(out, n->P, n->nparam * 4, kind_of(mem_kind, false), s);
    return cudaStreamSynchronize(s) == cudaSuccess ? HICARW_OK : HICARW_ERR_CUDA;
}

extern "C" int hicarw_unet_set_params(hicarw_unet *n, const float *in, int mem_kind, void *stream)
{
    api_entry();
    if (!n || !in) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemcpyAsync(n->P, in, n->nparam * 4, kind_of(mem_kind, true), s);
    pack_all(n, s);
    return cudaStreamSynchronize(s) == cudaSuccess ? HICARW_OK : HICARW_ERR_CUDA;
}

extern "C" int hicarw_unet_get_grads(hicarw_unet *n, float *out, int mem_kind, void *stream)
{
    api_entry();
    if (!n || !out) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemcpyAsync(out, n->Gr, n->nparam * 4, kind_of(mem_kind, false), s);
    return cudaStreamSynchronize(s) == cudaSuccess ? HICARW_OK : HICARW_ERR_CUDA;
}

extern "C" int hicarw_unet_zero_grads(hicarw_unet *n, void *stream)
{
    api_entry();
    if (!n) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(n->Gr, 0, n->nparam * 4, s);
    n->nsamples = 0;
    return cudaStreamSynchronize(s) == cudaSuccess ? HICARW_OK : HICARW_ERR_CUDA;
}

extern "C" int hicarw_unet_forward(hicarw_unet *n, const void *x0, float *out0, void *stream)
{
    api_entry();
    if (!n || !x0) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(n->err, 0, 4, s);
    int rc = unet_forward(n, (const uint4 *)x0, nullptr, s);
    if (out0) cudaMemcpyAsync(out0, n->O0, (size_t)n->nx[0] * n->ny[0] * n->nz * 4, cudaMemcpyDeviceToDevice, s);
    return finish(n, rc, s, "hicarw_unet_forward");
}

extern "C" int hicarw_unet_backward(hicarw_unet *n, const float *target, float weight, float *loss, void *stream)
{
    api_entry();
    if (!n || !target || !n->x_in) return HICARW_ERR_ARG;
    if (ensure_grads(n)) return HICARW_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(n->err, 0, 4, s);
    int rc = unet_backward(n, target, weight, s);
    if (loss) cudaMemcpyAsync(loss, n->scal + 2, 4, cudaMemcpyDeviceToHost, s);
    return finish(n, rc, s, "hicarw_unet_backward");
}

extern "C" int hicarw_unet_backward_residual(hicarw_unet *n, const float *coef, const float *rhat, float weight,
                                             float *loss, void *stream)
{
    api_entry();
    if (!n || !coef || !rhat || !n->x_in) return HICARW_ERR_ARG;
    if (ensure_grads(n)) return HICARW_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(n->err, 0, 4, s);
    int rc = unet_backward_residual(n, coef, rhat, weight, s);
    if (loss) cudaMemcpyAsync(loss, n->scal + 2, 4, cudaMemcpyDeviceToHost, s);
    return finish(n, rc, s, "hicarw_unet_backward_residual");
}

extern "C" int hicarw_unet_adam_step(hicarw_unet *n, float lr, void *stream)
{
    api_entry();
    if (!n || n->nsamples < 1) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    n->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)n->adam_t), c2 = 1.0f - powf(b2, (float)n->adam_t);
    unet_adam_kernel<<<ew_grid((long long)n->nparam), 256, 0, s>>>(n->P, n->Gr, n->M1, n->M2, (long long)n->nparam, lr,
                                                                   b1, b2, 1e-8f, c1, c2, 1.0f / n->nsamples);
    count_launch(1);
    pack_all(n, s);
    n->nsamples = 0;
    return cudaStreamSynchronize(s) == cudaSuccess ? HICARW_OK : HICARW_ERR_CUDA;
}

extern "C" int hicarw_unet_features(hicarw_unet *n, hicarw_handle *h, const double *r, void *x0, float *rms,
                                    void *stream)
{
    api_entry();
    if (!n || !h || !r || !x0) return HICARW_ERR_ARG;
    OpCtx c;
    handle_operator(h, &c);
    if (!c.probed || !unet_matches(n, c.d)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(n->err, 0, 4, s);
    const long long nvox = (long long)c.d.nx * c.d.ny * c.d.nz;
    feat_coef_kernel<<<ew_grid(nvox), 256, 0, s>>>(c, (uint4 *)x0, adim(n, 0, 16));
    unet_rms(n, c.d, r, plain_view(c.d), nullptr, s);
    feat_r_kernel<<<ew_grid(nvox), 256, 0, s>>>(r, plain_view(c.d), c.d, (uint4 *)x0, adim(n, 0, 16), n->scal, nullptr);
    count_launch(2);
    if (rms) cudaMemcpyAsync(rms, n->scal, 4, cudaMemcpyDeviceToHost, s);
    return finish(n, 0, s, "hicarw_unet_features");
}

extern "C" int hicarw_unet_apply(hicarw_unet *n, hicarw_handle *h, const double *r, double *z, void *stream)
{
    api_entry();
    if (!n || !h || !r || !z) return HICARW_ERR_ARG;
    OpCtx c;
    handle_operator(h, &c);
    if (!c.probed || !unet_matches(n, c.d)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(n->err, 0, 4, s);
    unet_prepare_operator(n, c, s);
    int rc = unet_apply(n, c, r, z, plain_view(c.d), nullptr, s);
    return finish(n, rc, s, "hicarw_unet_apply");
}

extern "C" int hicarw_nn_act_pitch(int nx) { return nx > 0 ? act_pitch(nx) : HICARW_ERR_ARG; }

// Run one convolution (or its data-gradient form) on caller-owned act-layout
// device tensors; synchronous on `stream`.
extern "C" int hicarw_nn_conv3(int cin, int cout, int nx, int ny, int nz, const void *in, const float *w,
                               const float *bias, const void *skip, const void *mask, int relu, int transpose, void *out,
                               float *out0, void *stream)
{
    api_entry();
    if (nx <= 0 || ny <= 0 || nz <= 0 || !in || !w || (!out && !out0)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int ci = transpose ? cout : cin, co = transpose ? cin : cout;
    uint4 *img = nullptr;
    int *err = nullptr;
    if (cudaMallocAsync((void **)&img, conv_wimage_bytes(cin, cout), s) != cudaSuccess) return HICARW_ERR_CUDA;
    if (cudaMallocAsync((void **)&err, sizeof(int), s) != cudaSuccess) {
        cudaFreeAsync(img, s);
        return HICARW_ERR_CUDA;
    }
    cudaMemsetAsync(err, 0, sizeof(int), s);
    if (transpose) conv_pack_bwd(w, cin, cout, img, s);
    else conv_pack_fwd(w, cin, cout, img, s);
    ConvArgs a{};
    a.in = (const uint4 *)in;
    a.out = (uint4 *)out;
    a.w = img;
    a.bias = bias;
    a.skip = (const uint4 *)skip;
    a.mask = (const uint4 *)mask;
    a.out0 = out0;
    a.din = act_dims(nx, ny, nz, ci);
    a.dout = act_dims(nx, ny, nz, co);
    a.relu = relu;
    a.err = err;
    a.gate = nullptr;
    int rc = conv3_fwd(ci, co, a, s);
    int herr = 0;
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(img, s);
    cudaFreeAsync(err, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (rc == -2) return HICARW_ERR_ARG;
    if (rc != 0 || e != cudaSuccess) {
        fprintf(stderr, "hicarw_nn_conv3: %s\n", cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError()));
        return HICARW_ERR_CUDA;
    }
    if (herr) {
        fprintf(stderr, "hicarw_nn_conv3: a pipeline wait timed out\n");
        return HICARW_ERR_CUDA;
    }
    return HICARW_OK;
}

// Mean duration (ms, CUDA events on `stream`) of `reps` forward launches of one
// convolution (bias + ReLU epilogue) on caller-owned act tensors, weights packed once.
extern "C" int hicarw_nn_conv3_time(int cin, int cout, int nx, int ny, int nz, const void *in, const float *w,
                                    const float *bias, void *out, int reps, void *stream, float *ms)
{
    api_entry();
    if (nx <= 0 || ny <= 0 || nz <= 0 || !in || !w || !out || reps < 1 || !ms) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    uint4 *img = nullptr;
    int *err = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc((void **)&img, conv_wimage_bytes(cin, cout)) != cudaSuccess) return HICARW_ERR_CUDA;
    if (cudaMalloc((void **)&err, sizeof(int)) != cudaSuccess) { cudaFree(img); return HICARW_ERR_CUDA; }
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(err, 0, sizeof(int), s);
    conv_pack_fwd(w, cin, cout, img, s);
    ConvArgs a{};
    a.in = (const uint4 *)in;
    a.out = (uint4 *)out;
    a.w = img;
    a.bias = bias;
    a.din = act_dims(nx, ny, nz, cin);
    a.dout = act_dims(nx, ny, nz, cout);
    a.relu = 1;
    a.err = err;
    int rc = conv3_fwd(cin, cout, a, s); // warm-up
    cudaEventRecord(e0, s);
    for (int q = 0; q < reps && rc == 0; q++) rc = conv3_fwd(cin, cout, a, s);
    cudaEventRecord(e1, s);
    int herr = 0;
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(img);
    cudaFree(err);
    if (rc == -2) return HICARW_ERR_ARG;
    if (rc != 0 || e != cudaSuccess || herr) return HICARW_ERR_CUDA;
    return HICARW_OK;
}

// Accumulate the weight and bias gradients of one convolution (caller zeroes dw, db).
extern "C" int hicarw_nn_conv3_wgrad(int cin, int cout, int nx, int ny, int nz, const void *x, const void *dy, float *dw,
                                     float *db, void *stream)
{
    api_entry();
    if (nx <= 0 || ny <= 0 || nz <= 0 || !x || !dy || !dw || !db) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int *err = nullptr;
    if (cudaMallocAsync((void **)&err, sizeof(int), s) != cudaSuccess) return HICARW_ERR_CUDA;
    cudaMemsetAsync(err, 0, sizeof(int), s);
    WgradArgs a{};
    a.x = (const uint4 *)x;
    a.dy = (const uint4 *)dy;
    a.dw = dw;
    a.db = db;
    a.dx = act_dims(nx, ny, nz, cin);
    a.ddy = act_dims(nx, ny, nz, cout);
    a.err = err;
    int rc = conv3_wgrad(cin, cout, a, s);
    int herr = 0;
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(err, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (rc == -2) return HICARW_ERR_ARG;
    if (rc != 0 || e != cudaSuccess) {
        fprintf(stderr, "hicarw_nn_conv3_wgrad: %s\n", cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError()));
        return HICARW_ERR_CUDA;
    }
    if (herr) {
        fprintf(stderr, "hicarw_nn_conv3_wgrad: a pipeline wait timed out\n");
        return HICARW_ERR_CUDA;
    }
    return HICARW_OK;
}
