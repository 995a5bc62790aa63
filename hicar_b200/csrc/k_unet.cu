// k_unet.cu -- C entry points of the tensor-core convolutions (k_conv.cu).
#include <cuda_runtime.h>
#include <stdio.h>

#include "../../include/hicarw.h"
#include "kernels.h"
#include "unet.h"

using namespace hw;

extern "C" int hicarw_nn_act_pitch(int nx) { return nx > 0 ? act_pitch(nx) : HICARW_ERR_ARG; }

// Run one convolution (or its data-gradient form) on caller-owned act-layout
// device tensors; synchronous on `stream`.
extern "C" int hicarw_nn_conv3(int cin, int cout, int nx, int ny, int nz, const void *in, const float *w,
                               const float *bias, const void *skip, const void *mask, int relu, int transpose, void *out,
                               float *out0, void *stream)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || !in || !w || (!out && !out0)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int ci = transpose ? cout : cin, co = transpose ? cin : cout;
    uint4 *img = nullptr;
    int *err = nullptr;
    if (cudaMallocAsync((void **)&img, conv_wimage_bytes(cin, cout), s) != cudaSuccess) return HICARW_ERR_CUDA;
    if (cudaMallocAsync((void **)&err, sizeof(int), s) != cudaSuccess) { cudaFreeAsync(img, s); return HICARW_ERR_CUDA; }
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
    if (herr) { fprintf(stderr, "hicarw_nn_conv3: a pipeline wait timed out\n"); return HICARW_ERR_CUDA; }
    return HICARW_OK;
}

// Accumulate the weight and bias gradients of one convolution (caller zeroes dw, db).
extern "C" int hicarw_nn_conv3_wgrad(int cin, int cout, int nx, int ny, int nz, const void *x, const void *dy, float *dw,
                                     float *db, void *stream)
{
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
    if (herr) { fprintf(stderr, "hicarw_nn_conv3_wgrad: a pipeline wait timed out\n"); return HICARW_ERR_CUDA; }
    return HICARW_OK;
}
