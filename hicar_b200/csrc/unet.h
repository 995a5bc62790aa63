// unet.h -- learned preconditioner: tensor-core 3x3x3 convolutions and the
// 3-level U-Net built from them (k_unet.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace hw {

// Activation layout of one U-Net level ("act layout"): BF16, channels in groups
// of 8 (16 bytes), one x-line per (j, k, group), lines padded by one zero cell
// on each side in x (i = -1 and i >= nx are zero) and one zero line of halo in
// j and k.  Element (c, i, k, j) lives at 16-byte unit
//     (((j+1)*(nz+2) + (k+1))*G + c/8)*PX + (i+1),   lane c%8,
// with PX = roundup(nx, 128) + 2 so that every 128-cell tile plus its halo is
// one contiguous 2080-byte run per channel group.
struct ActDims {
    int nx, ny, nz, G, PX;
};

__host__ __device__ inline int act_pitch(int nx) { return ((nx + 127) / 128) * 128 + 2; }
__host__ __device__ inline ActDims act_dims(int nx, int ny, int nz, int C)
{
    return ActDims{nx, ny, nz, C / 8, act_pitch(nx)};
}
__host__ __device__ inline long long act_units(const ActDims &a) // 16-byte units
{
    return (long long)(a.ny + 2) * (a.nz + 2) * a.G * a.PX;
}
__host__ __device__ inline long long act_unit(const ActDims &a, int i, int k, int j, int g)
{
    return (((long long)(j + 1) * (a.nz + 2) + (k + 1)) * a.G + g) * a.PX + (i + 1);
}

// One 3x3x3 "same" convolution launch on act-layout tensors.
//   out[v][co] = epilogue( bias[co] + sum_t sum_ci W[t][ci][co] in[v + off(t)][ci] )
// t = (dj+1)*9 + (dk+1)*3 + (di+1).  Epilogue, in order: + skip[v][co], ReLU,
// mask (zero where mask[v][co] <= 0).  out0 receives channel 0 in FP32 at the
// interior index (j*nz + k)*nx + i.
struct ConvArgs {
    const uint4 *in;
    uint4 *out;
    const uint4 *w; // packed BF16 weight image (conv_pack_*)
    const float *bias;
    const uint4 *skip;
    const uint4 *mask;
    float *out0;
    ActDims din, dout;
    int relu;
    int *err;
    const SolveState *gate; // kernels return at once when gate->stop (and not profiling)
};

// Weight gradient of one convolution: dw[t][ci][co] += sum_v dy[v][co] x[v + off(t)][ci],
// db[co] += sum_v dy[v][co] (dy is the gradient of the pre-activation output).
struct WgradArgs {
    const uint4 *x;
    const uint4 *dy;
    float *dw;
    float *db;
    ActDims dx, ddy;
    int *err;
};

size_t conv_wimage_bytes(int cin, int cout);
// BF16 image of W (FP32 [27][cin][cout]) for the forward conv cin -> cout
void conv_pack_fwd(const float *W, int cin, int cout, uint4 *img, cudaStream_t s);
// BF16 image of the data-gradient conv cout -> cin (flipped taps, transposed channels)
void conv_pack_bwd(const float *W, int cin, int cout, uint4 *img, cudaStream_t s);
int conv3_fwd(int cin, int cout, const ConvArgs &a, cudaStream_t s);
int conv3_wgrad(int cin, int cout, const WgradArgs &a, cudaStream_t s);

}  // namespace hw
