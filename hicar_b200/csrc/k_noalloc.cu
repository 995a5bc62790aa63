// k_noalloc.cu -- hicarw_residual_norm_noalloc: the FP64 residual norm
// ||rhs - A x||_2 of the handle's operator, for callers that cannot allocate.
//
// Some callers of this library cannot call cudaMalloc at the point where they
// want a residual check: code running inside a CUDA stream capture or a
// memory-pool-restricted region of a host model, or a Fortran time loop built
// around a preallocated OpenACC data region where any new device allocation
// is forbidden.  This entry point allocates nothing: its only scratch, one FP64
// partial sum per j-plane plus the arrival counter of the last-block
// reduction, lives in a file-scope __device__ array below, which every GPU
// that loads the library holds until the process exits.
//
// Limits and rules:
//  * at most NOALLOC_MAX_PLANES = 8192 j-planes (ny + 2 <= 8192); larger
//    grids are rejected with HICARW_ERR_ARG and a message;
//  * all calls share the array and it keeps the last call's contents: the
//    arrival counter is cleared (cudaMemsetAsync, no allocation) at the start
//    of every call, and calls that overlap on the GPU race on the array;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (a host-side name is not a device address); make that
//    first call before any stream capture.  The address is cached per device for
//    the life of the process, which assumes the device's primary context is not
//    reset (cudaDeviceReset) while the library is loaded.
#include <cuda_runtime.h>
#include <stdio.h>

#include <mutex>

#include "../../include/hicarw.h"
#include "common.cuh"
#include "kernels.h"

namespace hw {
// accessor of the handle's operator (capi.cu)
void handle_operator(const hicarw_handle *h, OpCtx *c);
void handle_set_error(hicarw_handle *h, const char *msg);
}  // namespace hw

using namespace hw;

constexpr int NOALLOC_MAX_PLANES = 8192;

struct NoallocScratch {
    double partial[NOALLOC_MAX_PLANES]; // one partial sum of squares per j-plane
    unsigned int arrived;               // CTAs that have published their partial
};

static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

// Residual of one row of the caller's unpadded (nx+2, nz+2, ny+2) FP64 arrays,
// the operator's coefficients read from the handle's padded layout.
__device__ __forceinline__ double noalloc_row(const OpCtx &c, const double *__restrict__ x, int i, int k, int j)
{
    const Dims &d = c.d;
    const long long sx = 1, sk = d.mx, sj = (long long)d.mx * d.mz;
    const long long q = i + sk * k + sj * j;
    if (i == 0 || i == d.mx - 1 || j == 0 || j == d.my - 1) return x[q];
    const long long N = d.npad;
    const float *cf = c.coef + kidx(d, i, k, j);
    if (c.probed) {
        if (k == 0 || k == d.mz - 1) return x[q];
        double y = (double)cf[CO * N] * x[q - sj - sk];
        y += (double)cf[CG * N] * x[q - sj];
        y += (double)cf[CM * N] * x[q - sj + sk];
        y += (double)cf[CK * N] * x[q - sk - sx];
        y += (double)cf[CC * N] * x[q - sk];
        y += (double)cf[CJ * N] * x[q - sk + sx];
        y += (double)cf[CE * N] * x[q - sx];
        y += (double)cf[CA * N] * x[q];
        y += (double)cf[CD * N] * x[q + sx];
        y += (double)cf[CI * N] * x[q + sk - sx];
        y += (double)cf[CB * N] * x[q + sk];
        y += (double)cf[CH * N] * x[q + sk + sx];
        y += (double)cf[CN * N] * x[q + sj - sk];
        y += (double)cf[CF * N] * x[q + sj];
        y += (double)cf[CL * N] * x[q + sj + sk];
        return y;
    }
    const BcCol b = c.bc[(long long)j * d.mx + i];
    if (k == d.mz - 1) return (x[q] - x[q - sk]) / b.dztop;
    if (k == 0) {
        double y = b.cy * x[q - sj];
        y += b.cy * x[q - sj + sk];
        y += b.cx * x[q - sx];
        y += b.m1 * x[q];
        y += (-b.cx) * x[q + sx];
        y += b.cx * x[q + sk - sx];
        y += b.p1 * x[q + sk];
        y += (-b.cx) * x[q + sk + sx];
        y += (-b.cy) * x[q + sj];
        y += (-b.cy) * x[q + sj + sk];
        return y;
    }
    const double dx = (double)d.dx;
    const double inv_dx2 = 1.0 / (dx * dx), neg4 = -4.0 * inv_dx2;
    const double bv = (double)cf[CB * N], cv = (double)cf[CC * N];
    double y = (double)cf[CO * N] * x[q - sj - sk];
    y += inv_dx2 * x[q - sj];
    y += (double)cf[CM * N] * x[q - sj + sk];
    y += (double)cf[CK * N] * x[q - sk - sx];
    y += cv * x[q - sk];
    y += (double)cf[CJ * N] * x[q - sk + sx];
    y += inv_dx2 * x[q - sx];
    y += (neg4 - bv - cv) * x[q];
    y += inv_dx2 * x[q + sx];
    y += (double)cf[CI * N] * x[q + sk - sx];
    y += bv * x[q + sk];
    y += (double)cf[CH * N] * x[q + sk + sx];
    y += (double)cf[CN * N] * x[q + sj - sk];
    y += inv_dx2 * x[q + sj];
    y += (double)cf[CL * N] * x[q + sj + sk];
    return y;
}

// One CTA per j-plane; the last CTA to arrive adds the plane partials in plane
// order and writes the norm.  Scratch comes from the caller-side lookup of
// g_noalloc_scratch (passed in as `scr`).
__global__ void __launch_bounds__(256) residual_norm_noalloc_kernel(OpCtx c, const double *__restrict__ x,
                                                                    const double *__restrict__ rhs,
                                                                    double *__restrict__ norm, NoallocScratch *scr)
{
    const Dims &d = c.d;
    const int j = blockIdx.x;
    const long long plane = (long long)d.mx * d.mz;
    double acc = 0.0;
    for (long long t = threadIdx.x; t < plane; t += blockDim.x) {
        int i = (int)(t % d.mx), k = (int)(t / d.mx);
        long long q = t + plane * j;
        double e = rhs[q] - noalloc_row(c, x, i, k, j);
        acc += e * e;
    }
    __shared__ double sh[8];
    __shared__ int last;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
        scr->partial[j] = s;
        __threadfence();
        unsigned int a = atomicAdd(&scr->arrived, 1u);
        last = (a == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double s = 0.0;
    for (int p = 0; p < (int)gridDim.x; p++) s += __ldcg(&scr->partial[p]);
    *norm = sqrt(s);
    scr->arrived = 0u;
}

// Per-device address of the scratch array, looked up once with the device current.
static std::mutex g_noalloc_mu;
static NoallocScratch *g_noalloc_addr[64] = {};

// Returns nullptr on success, else the reason the address could not be had.
static const char *noalloc_scratch(NoallocScratch **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return "cudaGetDevice failed";
    if (dev < 0 || dev >= 64) return "device index outside 0..63 (the per-device address cache has 64 entries)";
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) return "cudaGetSymbolAddress of the scratch array failed";
        g_noalloc_addr[dev] = (NoallocScratch *)p;
    }
    *out = g_noalloc_addr[dev];
    return nullptr;
}

extern "C" int hicarw_residual_norm_noalloc(hicarw_handle *h, const double *x, const double *rhs, double *norm,
                                            void *stream)
{
    api_entry();
    if (!h || !x || !rhs || !norm) return HICARW_ERR_ARG;
    OpCtx c;
    handle_operator(h, &c);
    if (c.d.my > NOALLOC_MAX_PLANES) {
        char msg[160];
        snprintf(msg, sizeof(msg), "hicarw_residual_norm_noalloc: ny + 2 = %d exceeds the %d j-planes of its "
                 "static scratch", c.d.my, NOALLOC_MAX_PLANES);
        handle_set_error(h, msg);
        return HICARW_ERR_ARG;
    }
    NoallocScratch *scr = nullptr;
    if (const char *why = noalloc_scratch(&scr)) {
        char msg[160];
        snprintf(msg, sizeof(msg), "hicarw_residual_norm_noalloc: %s", why);
        handle_set_error(h, msg);
        return HICARW_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(&scr->arrived, 0, sizeof(unsigned int), s) != cudaSuccess) {
        handle_set_error(h, "hicarw_residual_norm_noalloc: clearing the arrival counter failed");
        return HICARW_ERR_CUDA;
    }
    residual_norm_noalloc_kernel<<<c.d.my, 256, 0, s>>>(c, x, rhs, norm, scr);
    count_launch(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        handle_set_error(h, cudaGetErrorString(e));
        return HICARW_ERR_CUDA;
    }
    return HICARW_OK;
}
