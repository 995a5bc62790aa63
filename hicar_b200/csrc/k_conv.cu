// k_conv.cu -- 3x3x3 "same" convolutions on the 5th-generation tensor cores
// (tcgen05.mma kind::f16, BF16 operands, FP32 accumulators in tensor memory),
// used by the learned preconditioner.
//
// Forward (and data-gradient, with the flipped/transposed weight image) as an
// implicit GEMM: one 128-cell x-tile at (j, k) is D[128 x COUT] =
// sum over 27 taps and CIN/16 channel chunks of A_tap[128 x 16] * B_tap[COUT x 16]^T.
// The 9 neighbouring x-lines (dj, dk) of the tile, 130 cells each (one halo
// cell per side), are bulk-copied into shared memory with one 2080-byte copy per
// (line, channel group); in that no-swizzle K-major layout a tap's A operand is
// the line's matrix descriptor with the start address moved by (di+1) rows of
// 16 bytes, so the three x-shifts of a line share one copy.  The weight image is
// stored in global memory exactly as the B operands' shared-memory image and is
// bulk-copied once per CTA.  Persistent CTAs of 128 threads (one TMEM lane per
// thread) double-buffer the line stages: the copies of the next tile are in
// flight while the current tile's MMAs and epilogue run.
//
// Weight gradient: dW_tap[CIN x COUT] = sum over cells of X(v + tap)^T dY(v):
// the reduction runs over cells (the MMA's K), both operands MN-major straight
// from the same line images (8 cells x 8 channels = one 128-byte core matrix).
// Rows of one M=128 operand are 16 consecutive (line, channel group) blocks at
// the fixed 2080-byte line stride, so one descriptor covers several taps; the
// three x-shifts are three accumulators.  Each persistent CTA accumulates all of
// its tiles in TMEM and adds its partial sums to the FP32 gradient at the end.
#include <cuda_bf16.h>
#include <stdio.h>

#include "kernels.h"
#include "tc05.cuh"
#include "unet.h"

namespace hw {

constexpr int TILE = 128;
constexpr int LROWS = TILE + 2;
constexpr int LG = LROWS * 16; // bytes of one (line, channel group) image with halo
constexpr int YG = TILE * 16;  // bytes of one (line, channel group) image without halo

__device__ __forceinline__ bool conv_gated(const SolveState *g)
{
    return g && *(volatile const int *)&g->stop != 0 && !g->profile;
}

__device__ __forceinline__ void unpack8(const uint4 &u, float (&f)[8])
{
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float2 t = __bfloat1622float2(h[q]);
        f[2 * q] = t.x;
        f[2 * q + 1] = t.y;
    }
}

__device__ __forceinline__ uint4 pack8(const float *f)
{
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
    return u;
}

template <int CIN, int COUT>
struct FwdCfg {
    static constexpr int GI = CIN / 8, GO = COUT / 8;
    static constexpr int WB = 27 * GI * COUT * 16; // weight image bytes
    static constexpr int STAGE = 9 * GI * LG;      // one tile's line images
    static constexpr int NCOL = 2 * COUT <= 32 ? 32 : (2 * COUT <= 64 ? 64 : 128);
    static constexpr int SMEM = WB + 2 * STAGE + 64;
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 128, "channel counts");
    static_assert(SMEM <= 232448, "shared memory");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) conv3_fwd_kernel(ConvArgs a)
{
    using C = FwdCfg<CIN, COUT>;
    if (conv_gated(a.gate)) return;
    extern __shared__ __align__(128) uint8_t sm[];
    uint8_t *wsm = sm;
    uint8_t *stg0 = sm + C::WB, *stg1 = sm + C::WB + C::STAGE;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + C::WB + 2 * C::STAGE); // copy[0], copy[1], mma[0], mma[1]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 4);
    const int tid = threadIdx.x, warp = tid >> 5;
    const ActDims di = a.din, dd = a.dout;
    const int ntx = (di.nx + TILE - 1) / TILE;
    const int ntiles = ntx * di.nz * di.ny;
    if (tid == 0) {
        for (int q = 0; q < 4; q++) tc::mbar_init(&bars[q], 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(tslot, C::NCOL);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    const char *inb = reinterpret_cast<const char *>(a.in);

    // called by all lanes of warp 0: lane 0 posts the byte count, then the lanes
    // issue one bulk copy each
    auto issue = [&](int tile, int s, bool with_w) {
        const int tx = tile % ntx, r = tile / ntx, k = r % di.nz, j = r / di.nz;
        const int lane = tid & 31;
        uint8_t *dst = s ? stg1 : stg0;
        if (lane == 0) tc::mbar_expect_tx(&bars[s], C::STAGE + (with_w ? C::WB : 0));
        __syncwarp();
        if (with_w && lane == 31) tc::bulk_g2s(wsm, a.w, C::WB, &bars[s]);
        for (int q = lane; lane < 31 && q < 9 * C::GI; q += 31) { // lanes 0..30: the line images
            const int sl = q / C::GI, g = q % C::GI;
            const long long L = (long long)(j + sl / 3) * (di.nz + 2) + (k + sl % 3); // line (j+dj+1, k+dk+1)
            tc::bulk_g2s(dst + (sl * C::GI + g) * LG, inb + ((L * C::GI + g) * di.PX + (long long)tx * TILE) * 16, LG,
                         &bars[s]);
        }
    };

    constexpr uint32_t IDESC = tc::idesc_bf16(128, COUT, 0, 0);
    // Pipeline: in iteration `it` the MMAs of tile `it` (TMEM buffer it&1) run
    // while the epilogue of tile it-1 (buffer (it-1)&1) reads the other buffer,
    // and the copies of tile it+1 go into the line stage that tile it-1 used,
    // issued as soon as its MMAs have completed.  mbarriers: [0], [1] line
    // stages, [2], [3] MMA completion per TMEM buffer.
    bool ok = true;
    int it = 0, tile = blockIdx.x, prev = -1;
    if (warp == 0 && tile < ntiles) issue(tile, 0, true);
    for (;; it++) {
        const bool have = tile < ntiles;
        const int s = it & 1;
        if (have) {
            const bool got = tc::mbar_wait(&bars[s], (it >> 1) & 1);
            if (!__syncthreads_and(got)) { ok = false; break; }
            if (tid == 0) {
                tc::fence_after();
                // descriptors of the stage / weight bases; every operand is a
                // compile-time byte offset from them (start field = address >> 4)
                const uint64_t a0 = tc::sdesc(tc::smem_u32(s ? stg1 : stg0), LG, 128);
                const uint64_t b0 = tc::sdesc(tc::smem_u32(wsm), COUT * 16, 128);
#pragma unroll
                for (int t = 0; t < 27; t++) {
#pragma unroll
                    for (int c = 0; c < C::GI / 2; c++) {
                        const uint64_t ad = a0 + (uint64_t)((((t / 3) * C::GI + 2 * c) * LG + (t % 3) * 16) >> 4);
                        const uint64_t bd = b0 + (uint64_t)(((t * C::GI + 2 * c) * COUT * 16) >> 4);
                        tc::mma_bf16(tmem + s * COUT, ad, bd, IDESC, (t | c) ? 1u : 0u);
                    }
                }
                tc::mma_commit(&bars[2 + s]);
            }
        }
        const int nxt = have ? tile + (int)gridDim.x : ntiles;
        if (it == 0) {
            if (warp == 0 && nxt < ntiles) issue(nxt, s ^ 1, false); // stage 1 not used yet
        } else {
            // tile it-1: its MMAs done -> its line stage is free, its accumulator readable
            const bool done = tc::mbar_wait(&bars[2 + (s ^ 1)], ((it - 1) >> 1) & 1);
            if (!__syncthreads_and(done)) { ok = false; break; }
            if (warp == 0 && nxt < ntiles) issue(nxt, s ^ 1, false);
            tc::fence_after();
            const int tx = prev % ntx, r = prev / ntx, k = r % di.nz, j = r / di.nz;
            const int i = tx * TILE + tid;
            const uint32_t acc_col = (uint32_t)((s ^ 1) * COUT);
            float v[COUT];
#pragma unroll
            for (int q = 0; q < COUT / 16; q++) {
                float t16[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + acc_col + (uint32_t)(q * 16), t16);
#pragma unroll
                for (int e = 0; e < 16; e++) v[q * 16 + e] = t16[e];
            }
            if (i < di.nx) {
                if (a.bias) {
#pragma unroll
                    for (int c = 0; c < COUT; c++) v[c] += __ldg(a.bias + c);
                }
                if (a.skip) {
#pragma unroll
                    for (int g = 0; g < C::GO; g++) {
                        float f[8];
                        unpack8(a.skip[act_unit(dd, i, k, j, g)], f);
#pragma unroll
                        for (int e = 0; e < 8; e++) v[g * 8 + e] += f[e];
                    }
                }
                if (a.relu) {
#pragma unroll
                    for (int c = 0; c < COUT; c++) v[c] = fmaxf(v[c], 0.0f);
                }
                if (a.mask) {
#pragma unroll
                    for (int g = 0; g < C::GO; g++) {
                        float f[8];
                        unpack8(a.mask[act_unit(dd, i, k, j, g)], f);
#pragma unroll
                        for (int e = 0; e < 8; e++) v[g * 8 + e] = f[e] > 0.0f ? v[g * 8 + e] : 0.0f;
                    }
                }
                if (a.out) {
#pragma unroll
                    for (int g = 0; g < C::GO; g++) a.out[act_unit(dd, i, k, j, g)] = pack8(v + g * 8);
                }
                if (a.out0) a.out0[((long long)j * dd.nz + k) * dd.nx + i] = v[0];
            }
        }
        tc::fence_before();
        __syncthreads();
        if (!have) break;
        prev = tile;
        tile = nxt;
    }
    if (!ok && tid == 0) {
        atomicExch(a.err, 1);
        // bounded waits for the copies and MMAs this CTA may still have in flight
        for (int q = 0; q < 4; q++) tc::mbar_wait(&bars[q], (uint32_t)(q < 2 ? (it >> 1) & 1 : (it & 1)), 100000000ull);
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, C::NCOL);
}

template <int CIN, int COUT>
struct WgCfg {
    static constexpr int GI = CIN / 8, GO = COUT / 8;
    static constexpr int NB = 9 * GI;          // (line, channel group) blocks of one x-shift
    static constexpr int NMC = (NB + 15) / 16; // M = 128 row chunks
    static constexpr int XR = NMC * 16 * LG;   // input lines + slack read by the last chunk
    static constexpr int YR = GO * YG;
    static constexpr int STAGE = XR + YR;
    static constexpr int NACC = 3 * NMC;
    static constexpr int NEED = NACC * COUT;
    static constexpr int NCOL = NEED <= 32 ? 32 : NEED <= 64 ? 64 : NEED <= 128 ? 128 : NEED <= 256 ? 256 : 512;
    static constexpr int SMEM = 2 * STAGE + 64;
    static_assert(NEED <= 512, "tensor memory columns");
    static_assert(SMEM <= 232448, "shared memory");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) conv3_wgrad_kernel(WgradArgs a)
{
    using C = WgCfg<CIN, COUT>;
    extern __shared__ __align__(128) uint8_t sm[];
    uint8_t *stg0 = sm, *stg1 = sm + C::STAGE;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + 2 * C::STAGE);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 3);
    const int tid = threadIdx.x, warp = tid >> 5;
    const ActDims dx = a.dx, dy = a.ddy;
    const int ntx = (dx.nx + TILE - 1) / TILE;
    const int ntiles = ntx * dx.nz * dx.ny;
    if (tid == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        tc::mbar_init(&bars[2], 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(tslot, C::NCOL);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    const char *xb = reinterpret_cast<const char *>(a.x);
    const char *yb = reinterpret_cast<const char *>(a.dy);

    // called by all lanes of warp 0 (see the forward kernel)
    auto issue = [&](int tile, int s) {
        const int tx = tile % ntx, r = tile / ntx, k = r % dx.nz, j = r / dx.nz;
        const int lane = tid & 31;
        uint8_t *dst = s ? stg1 : stg0;
        if (lane == 0) tc::mbar_expect_tx(&bars[s], 9 * C::GI * LG + C::YR);
        __syncwarp();
        for (int q = lane; q < 9 * C::GI + C::GO; q += 32) {
            if (q < 9 * C::GI) {
                const int sl = q / C::GI, g = q % C::GI;
                const long long L = (long long)(j + sl / 3) * (dx.nz + 2) + (k + sl % 3);
                tc::bulk_g2s(dst + (sl * C::GI + g) * LG, xb + ((L * C::GI + g) * dx.PX + (long long)tx * TILE) * 16,
                             LG, &bars[s]);
            } else {
                const int g = q - 9 * C::GI;
                const long long L0 = (long long)(j + 1) * (dy.nz + 2) + (k + 1);
                tc::bulk_g2s(dst + C::XR + g * YG, yb + ((L0 * C::GO + g) * dy.PX + (long long)tx * TILE + 1) * 16,
                             YG, &bars[s]);
            }
        }
    };

    constexpr uint32_t IDESC = tc::idesc_bf16(128, COUT, 1, 1);
    float db[COUT];
#pragma unroll
    for (int c = 0; c < COUT; c++) db[c] = 0.0f;
    bool ok = true;
    int it = 0, tile = blockIdx.x;
    if (warp == 0 && tile < ntiles) issue(tile, 0);
    for (; tile < ntiles; tile += gridDim.x, it++) {
        const int s = it & 1;
        if (warp == 0 && tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x, s ^ 1);
        const bool got = tc::mbar_wait(&bars[s], (it >> 1) & 1);
        if (!__syncthreads_and(got)) { ok = false; break; }
        const uint8_t *st = s ? stg1 : stg0;
        if (tid == 0) {
            tc::fence_after();
            const uint64_t a0 = tc::sdesc(tc::smem_u32(st), 128, LG);
            const uint64_t b0 = tc::sdesc(tc::smem_u32(st) + C::XR, 128, YG);
#pragma unroll
            for (int dil = 0; dil < 3; dil++)
#pragma unroll
                for (int mc = 0; mc < C::NMC; mc++) {
                    const uint32_t d = tmem + (uint32_t)((dil * C::NMC + mc) * COUT);
#pragma unroll
                    for (int kc = 0; kc < TILE / 16; kc++) {
                        const uint64_t ad = a0 + (uint64_t)((mc * 16 * LG + dil * 16 + kc * 256) >> 4);
                        const uint64_t bd = b0 + (uint64_t)((kc * 256) >> 4);
                        tc::mma_bf16(d, ad, bd, IDESC, (it > 0 || kc > 0) ? 1u : 0u);
                    }
                }
            tc::mma_commit(&bars[2]);
        }
        // bias gradient: this thread's cell row of dy
#pragma unroll
        for (int g = 0; g < C::GO; g++) {
            float f[8];
            unpack8(*reinterpret_cast<const uint4 *>(st + C::XR + g * YG + tid * 16), f);
#pragma unroll
            for (int e = 0; e < 8; e++) db[g * 8 + e] += f[e];
        }
        const bool done = tc::mbar_wait(&bars[2], it & 1);
        if (!__syncthreads_and(done)) { ok = false; break; }
        tc::fence_before();
        __syncthreads();
    }
    if (ok && it > 0) {
        tc::fence_after();
        for (int dil = 0; dil < 3; dil++)
            for (int mc = 0; mc < C::NMC; mc++)
#pragma unroll
                for (int q = 0; q < COUT / 16; q++) {
                    float v[16];
                    tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) +
                                      (uint32_t)((dil * C::NMC + mc) * COUT + q * 16),
                                  v);
                    const int b = mc * 16 + tid / 8;
                    if (b < C::NB) {
                        const int sl = b / C::GI, g = b % C::GI, ci = g * 8 + (tid & 7), t = sl * 3 + dil;
                        float *dst = a.dw + ((long long)t * CIN + ci) * COUT + q * 16;
#pragma unroll
                        for (int e = 0; e < 16; e++) atomicAdd(dst + e, v[e]);
                    }
                }
#pragma unroll
        for (int c = 0; c < COUT; c++) {
            float x = db[c];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if ((tid & 31) == 0) atomicAdd(a.db + c, x);
        }
    }
    if (!ok && tid == 0) {
        atomicExch(a.err, 1);
        tc::mbar_wait(&bars[0], 0, 100000000ull);
        tc::mbar_wait(&bars[1], 0, 100000000ull);
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, C::NCOL);
}

// ---------------------------------------------------------------------------
__global__ void conv_pack_fwd_kernel(const float *__restrict__ W, int cin, int cout, __nv_bfloat16 *__restrict__ img)
{
    const int n = 27 * cin * cout;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int t = q / (cin * cout), r = q % (cin * cout), ci = r / cout, co = r % cout;
        img[(((long long)t * (cin / 8) + ci / 8) * cout + co) * 8 + (ci & 7)] = __float2bfloat16_rn(W[q]);
    }
}

// image of the conv cout -> cin whose output is the data gradient:
// W'[t'][ci' = co][co' = ci] = W[26 - t'][ci][co]
__global__ void conv_pack_bwd_kernel(const float *__restrict__ W, int cin, int cout, __nv_bfloat16 *__restrict__ img)
{
    const int n = 27 * cin * cout;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int t = q / (cin * cout), r = q % (cin * cout), ci = r / cout, co = r % cout;
        const int tf = 26 - t;
        img[(((long long)tf * (cout / 8) + co / 8) * cin + ci) * 8 + (co & 7)] = __float2bfloat16_rn(W[q]);
    }
}

size_t conv_wimage_bytes(int cin, int cout) { return (size_t)27 * cin * cout * 2; }

void conv_pack_fwd(const float *W, int cin, int cout, uint4 *img, cudaStream_t s)
{
    conv_pack_fwd_kernel<<<(27 * cin * cout + 255) / 256, 256, 0, s>>>(W, cin, cout, (__nv_bfloat16 *)img);
    count_launch(1);
}

void conv_pack_bwd(const float *W, int cin, int cout, uint4 *img, cudaStream_t s)
{
    conv_pack_bwd_kernel<<<(27 * cin * cout + 255) / 256, 256, 0, s>>>(W, cin, cout, (__nv_bfloat16 *)img);
    count_launch(1);
}

static int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

template <int CI, int CO>
static int launch_fwd(const ConvArgs &a, cudaStream_t s)
{
    using C = FwdCfg<CI, CO>;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(conv3_fwd_kernel<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM) !=
            cudaSuccess)
            return -1;
        attr = true;
    }
    const long long ntiles = (long long)((a.din.nx + TILE - 1) / TILE) * a.din.nz * a.din.ny;
    const int per_sm = C::SMEM <= 113 * 1024 ? 2 : 1;
    const int grid = (int)(ntiles < (long long)sm_count() * per_sm ? ntiles : (long long)sm_count() * per_sm);
    if (grid <= 0) return 0;
    char name[32];
    snprintf(name, sizeof(name), "conv3_fwd_%dx%d", CI, CO);
    const double cells = (double)a.din.nx * a.din.ny * a.din.nz;
    ProfScope ps_(name, cells * 2.0 * (CI + CO), s);
    conv3_fwd_kernel<CI, CO><<<grid, 128, C::SMEM, s>>>(a);
    count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <int CI, int CO>
static int launch_wgrad(const WgradArgs &a, cudaStream_t s)
{
    using C = WgCfg<CI, CO>;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(conv3_wgrad_kernel<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM) !=
            cudaSuccess)
            return -1;
        attr = true;
    }
    const long long ntiles = (long long)((a.dx.nx + TILE - 1) / TILE) * a.dx.nz * a.dx.ny;
    const int grid = (int)(ntiles < sm_count() ? ntiles : sm_count()); // 1 CTA per SM (TMEM / smem)
    if (grid <= 0) return 0;
    char name[32];
    snprintf(name, sizeof(name), "conv3_wgrad_%dx%d", CI, CO);
    const double cells = (double)a.dx.nx * a.dx.ny * a.dx.nz;
    ProfScope ps_(name, cells * 2.0 * (CI + CO), s);
    conv3_wgrad_kernel<CI, CO><<<grid, 128, C::SMEM, s>>>(a);
    count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static bool dims_ok(const ActDims &a, int C)
{
    return a.nx > 0 && a.ny > 0 && a.nz > 0 && a.G * 8 == C && a.PX == act_pitch(a.nx);
}

int conv3_fwd(int cin, int cout, const ConvArgs &a, cudaStream_t s)
{
    if (!dims_ok(a.din, cin) || !dims_ok(a.dout, cout) || a.din.nx != a.dout.nx || a.din.ny != a.dout.ny ||
        a.din.nz != a.dout.nz || !a.in || !a.w || !a.err)
        return -2;
    if (!aligned16(a.in) || !aligned16(a.w) || !aligned16(a.out) || !aligned16(a.skip) || !aligned16(a.mask)) return -2;
    if (cin == 16 && cout == 16) return launch_fwd<16, 16>(a, s);
    if (cin == 16 && cout == 32) return launch_fwd<16, 32>(a, s);
    if (cin == 32 && cout == 32) return launch_fwd<32, 32>(a, s);
    if (cin == 32 && cout == 16) return launch_fwd<32, 16>(a, s);
    return -2;
}

int conv3_wgrad(int cin, int cout, const WgradArgs &a, cudaStream_t s)
{
    if (!dims_ok(a.dx, cin) || !dims_ok(a.ddy, cout) || a.dx.nx != a.ddy.nx || a.dx.ny != a.ddy.ny ||
        a.dx.nz != a.ddy.nz || !a.x || !a.dy || !a.dw || !a.db || !a.err)
        return -2;
    if (!aligned16(a.x) || !aligned16(a.dy)) return -2;
    if (cin == 16 && cout == 16) return launch_wgrad<16, 16>(a, s);
    if (cin == 16 && cout == 32) return launch_wgrad<16, 32>(a, s);
    if (cin == 32 && cout == 32) return launch_wgrad<32, 32>(a, s);
    if (cin == 32 && cout == 16) return launch_wgrad<32, 16>(a, s);
    return -2;
}

}  // namespace hw
