// k_model.cu -- the model-side FP32 arithmetic of the wind solve:
//   * calc_divergence (wind.F90:250-523)                         -> divergence_kernel
//   * calc_updated_winds (wind_iterative.F90:1742-2071)            -> winds_kernel
//   * probe_lambda_pattern / probe_record (:1096-1115, :1169-1231) -> probe_* kernels
//   * init_module_vars (:2274-2421), initialize_coefs + update_coefs_host
//     (:2424-2552), update_coefs_gpu (:2555-2603)                  -> coefficient kernels
//   * extract_diagonal (:1041-1075), compute_rhs_3d (:1513-1530)
//
// This file is compiled with -fmad=false: every FP32 multiply and add is rounded
// separately and evaluated in the reference's left-to-right order, so the
// probed operator A = 2 D o G comes out bit-identical to a CPU evaluation of the
// same statements.  Each output element is produced by one thread; the
// neighbouring face values a cell needs are recomputed rather than staged,
// which keeps every kernel a single coalesced pass along i.
#include "common.cuh"
#include "kernels.h"

namespace hw {

// ---------------------------------------------------------------------------
// calc_divergence, one thread per cell (i, k, j).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float u_met(const Dims &d, const Metrics &m, const float *u, const float *rho, int i, int k,
                                       int j, int adv_den, int use_dqdt)
{
    long long q = uidx(d, i, k, j);
    if (adv_den) {
        if (i == 1) return u[q] * m.ju[q] * (1.5f * rho[cidx(d, 1, k, j)] - 0.5f * rho[cidx(d, 2, k, j)]);
        if (i == d.nx + 1) return u[q] * m.ju[q] * (1.5f * rho[cidx(d, d.nx, k, j)] - 0.5f * rho[cidx(d, d.nx - 1, k, j)]);
        return u[q] * m.ju[q] * (rho[cidx(d, i - 1, k, j)] + rho[cidx(d, i, k, j)]) / 2.0f;
    }
    return use_dqdt ? u[q] : u[q] * m.ju[q];
}

__device__ __forceinline__ float v_met(const Dims &d, const Metrics &m, const float *v, const float *rho, int i, int k,
                                       int j, int adv_den, int use_dqdt)
{
    long long q = cidx(d, i, k, j);
    if (adv_den) {
        if (j == 1) return v[q] * m.jv[q] * (1.5f * rho[cidx(d, i, k, 1)] - 0.5f * rho[cidx(d, i, k, 2)]);
        if (j == d.ny + 1) return v[q] * m.jv[q] * (1.5f * rho[cidx(d, i, k, d.ny)] - 0.5f * rho[cidx(d, i, k, d.ny - 1)]);
        return v[q] * m.jv[q] * (rho[cidx(d, i, k, j - 1)] + rho[cidx(d, i, k, j)]) / 2.0f;
    }
    return use_dqdt ? v[q] : v[q] * m.jv[q];
}

__device__ __forceinline__ float w_met(const Dims &d, const Metrics &m, const float *w, const float *rho, int i, int k,
                                       int j, int adv_den)
{
    long long c = cidx(d, i, k, j);
    if (adv_den) {
        if (k < d.nz) {
            long long cp = cidx(d, i, k + 1, j);
            float rho_i = (rho[c] * m.adz[cp] + rho[cp] * m.adz[c]) / (m.adz[c] + m.adz[cp]);
            return w[c] * m.jw[c] * rho_i;
        }
        return w[c] * m.jw[c] * rho[c];
    }
    return w[c] * m.jw[c];
}

__global__ void divergence_kernel(Dims d, Metrics m, const float *__restrict__ u, const float *__restrict__ v,
                                  const float *__restrict__ w, const float *__restrict__ rho, float *__restrict__ div,
                                  int adv_den, int horz_only, int use_dqdt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1;
    int j = blockIdx.z + 1;
    if (i > d.nx) return;
    float um1 = u_met(d, m, u, rho, i + 1, k, j, adv_den, use_dqdt);
    float um0 = u_met(d, m, u, rho, i, k, j, adv_den, use_dqdt);
    float vm1 = v_met(d, m, v, rho, i, k, j + 1, adv_den, use_dqdt);
    float vm0 = v_met(d, m, v, rho, i, k, j, adv_den, use_dqdt);
    float sum = um1 / m.mf_my_u[i2u(d, i + 1, j)] - um0 / m.mf_my_u[i2u(d, i, j)] + vm1 / m.mf_mx_v[i2(d, i, j + 1)] -
                vm0 / m.mf_mx_v[i2(d, i, j)];
    float dv = m.mf_mxy[i2(d, i, j)] * sum / d.dx;
    if (!horz_only) {
        long long c = cidx(d, i, k, j);
        float wk = w_met(d, m, w, rho, i, k, j, adv_den);
        if (k == 1) dv = dv + wk / (m.adz[c]);
        else dv = dv + (wk - w_met(d, m, w, rho, i, k - 1, j, adv_den)) / (m.adz[c]);
        dv = dv / m.jac[c];
    }
    div[cidx(d, i, k, j)] = dv;
}

void launch_divergence(const Dims &d, const Metrics &m, const float *u, const float *v, const float *w,
                       const float *rho, float *div, int adv_den, int horz_only, int use_dqdt, cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.nz, d.ny);
    divergence_kernel<<<g, b, 0, st>>>(d, m, u, v, w, rho, div, adv_den, horz_only, use_dqdt);
    count_launch(1);
}

// ---------------------------------------------------------------------------
// calc_updated_winds: one thread per (i, k, j) of the (nx+1) x nz x (ny+1) box;
// it updates the u face (i,k,j) when j <= ny, the v face when i <= nx, and
// w_grid at (i,k,j) when i <= nx, j <= ny, k <= nz-1 (rigid lid at k_e).
// ---------------------------------------------------------------------------
template <typename V>
__device__ __forceinline__ float lam(const Dims &d, const V *x, int i, int k, int j)
{
    return (float)x[kidx(d, i, k, j)]; // lambda_3d = real(x_sol) (:1775-1781)
}

template <typename V>
__global__ void winds_kernel(Dims d, Metrics m, const V *__restrict__ x, const float *__restrict__ alpha,
                             const float *__restrict__ rho, float *__restrict__ u, float *__restrict__ v,
                             float *__restrict__ w, int adv_den)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1;
    int j = blockIdx.z + 1;
    if (i > d.nx + 1) return;
    const int nz = d.nz;
    const float dzk1 = m.dz_if[zidx(d, 1, 2, 1)];
    const float dzke = m.dz_if[zidx(d, 1, nz, 1)];
    const float den = m.dz_if[zidx(d, 1, k + 1, 1)] + m.dz_if[zidx(d, 1, k, 1)];
    if (j <= d.ny) { // u face (:1948-1954, :1964-1970, :1984-1990, :2004-2013)
        float dl;
        if (k == nz) dl = ((lam(d, x, i, nz, j) + lam(d, x, i - 1, nz, j)) / 2.0f - (lam(d, x, i, nz - 1, j) + lam(d, x, i - 1, nz - 1, j)) / 2.0f) / dzke;
        else if (k == 1) dl = ((lam(d, x, i, 2, j) + lam(d, x, i - 1, 2, j)) / 2.0f - (lam(d, x, i, 1, j) + lam(d, x, i - 1, 1, j)) / 2.0f) / dzk1;
        else {
            float t = (lam(d, x, i, k + 1, j) + lam(d, x, i - 1, k + 1, j)) / 2.0f - (lam(d, x, i, k - 1, j) + lam(d, x, i - 1, k - 1, j)) / 2.0f;
            dl = t / den;
        }
        float rho_u;
        if (!adv_den) rho_u = 1.0f;
        else if (i == 1) rho_u = rho[cidx(d, 1, k, j)];
        else if (i == d.nx + 1) rho_u = rho[cidx(d, d.nx, k, j)];
        else rho_u = 0.5f * (rho[cidx(d, i, k, j)] + rho[cidx(d, i - 1, k, j)]);
        long long q = uidx(d, i, k, j);
        float grad = (lam(d, x, i, k, j) - lam(d, x, i - 1, k, j)) / d.dx - m.dzdx_u[q] * (dl) / m.ju[q];
        u[q] = u[q] + 0.5f * m.mf_mx_u[i2u(d, i, j)] * grad / (rho_u);
    }
    if (i <= d.nx) { // v face (:1956-1962, :1972-1978, :1991-1997, :2015-2024)
        float dl;
        if (k == nz) dl = ((lam(d, x, i, nz, j) + lam(d, x, i, nz, j - 1)) / 2.0f - (lam(d, x, i, nz - 1, j) + lam(d, x, i, nz - 1, j - 1)) / 2.0f) / dzke;
        else if (k == 1) dl = ((lam(d, x, i, 2, j) + lam(d, x, i, 2, j - 1)) / 2.0f - (lam(d, x, i, 1, j) + lam(d, x, i, 1, j - 1)) / 2.0f) / dzk1;
        else {
            float t = (lam(d, x, i, k + 1, j) + lam(d, x, i, k + 1, j - 1)) / 2.0f - (lam(d, x, i, k - 1, j) + lam(d, x, i, k - 1, j - 1)) / 2.0f;
            dl = t / den;
        }
        float rho_v;
        if (!adv_den) rho_v = 1.0f;
        else if (j == 1) rho_v = rho[cidx(d, i, k, 1)];
        else if (j == d.ny + 1) rho_v = rho[cidx(d, i, k, d.ny)];
        else rho_v = 0.5f * (rho[cidx(d, i, k, j)] + rho[cidx(d, i, k, j - 1)]);
        long long q = cidx(d, i, k, j);
        float grad = (lam(d, x, i, k, j) - lam(d, x, i, k, j - 1)) / d.dx - m.dzdy_v[q] * (dl) / m.jv[q];
        v[q] = v[q] + 0.5f * m.mf_my_v[i2(d, i, j)] * grad / (rho_v);
    }
    if (i <= d.nx && j <= d.ny && k <= nz - 1) { // w_grid (:2038-2050)
        long long c = cidx(d, i, k, j);
        float rho_w = 1.0f;
        if (adv_den) {
            long long cp = cidx(d, i, k + 1, j);
            rho_w = (rho[c] * m.adz[cp] + rho[cp] * m.adz[c]) / (m.adz[c] + m.adz[cp]);
        }
        float a = alpha[c];
        w[c] = w[c] + 0.5f * (a * a) * (lam(d, x, i, k + 1, j) - lam(d, x, i, k, j)) / m.dz_if[zidx(d, i, k + 1, j)] / m.jw[c] / rho_w;
    }
}

template <typename V>
void launch_winds(const Dims &d, const Metrics &m, const V *x, const float *alpha, const float *rho, float *u, float *v,
                  float *w, int adv_den, cudaStream_t st)
{
    dim3 b(128), g((d.nx + 1 + 127) / 128, d.nz, d.ny + 1);
    winds_kernel<V><<<g, b, 0, st>>>(d, m, x, alpha, rho, u, v, w, adv_den);
    count_launch(1);
}
template void launch_winds<double>(const Dims &, const Metrics &, const double *, const float *, const float *, float *,
                                   float *, float *, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Probing (:1096-1248).
// ---------------------------------------------------------------------------
template <typename V>
__global__ void probe_pattern_kernel(Dims d, V *x, int ca, int cb, int cc)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int k = blockIdx.y, j = blockIdx.z;
    if (i >= d.mx) return;
    bool on = i >= 1 && i <= d.mx - 2 && k >= 1 && k <= d.mz - 2 && j >= 1 && j <= d.my - 2 && i % 3 == ca &&
              k % 3 == cb && j % 3 == cc;
    x[kidx(d, i, k, j)] = on ? (V)1 : (V)0;
}

template <typename V>
void launch_probe_pattern(const Dims &d, V *x, int ca, int cb, int cc, cudaStream_t st)
{
    dim3 b(128), g((d.mx + 127) / 128, d.mz, d.my);
    probe_pattern_kernel<V><<<g, b, 0, st>>>(d, x, ca, cb, cc);
    count_launch(1);
}
template void launch_probe_pattern<double>(const Dims &, double *, int, int, int, cudaStream_t);

__global__ void probe_record_kernel(Dims d, const float *__restrict__ T, float *coef, int ca, int cb, int cc,
                                    unsigned int *max_leak_bits)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1, j = blockIdx.z + 1;
    float leak = 0.0f;
    if (i <= d.nx) {
        int di = (ca - i % 3 + 3) % 3; if (di == 2) di = -1;
        int dk = (cb - k % 3 + 3) % 3; if (dk == 2) dk = -1;
        int dj = (cc - j % 3 + 3) % 3; if (dj == 2) dj = -1;
        float tv = 2.0f * T[cidx(d, i, k, j)];
        int slot = -1;
        if (dk == 0) {
            if (di == 0 && dj == 0) slot = CA; else if (di == 1 && dj == 0) slot = CD; else if (di == -1 && dj == 0) slot = CE;
            else if (di == 0 && dj == 1) slot = CF; else if (di == 0 && dj == -1) slot = CG;
        } else if (dk == 1) {
            if (di == 0 && dj == 0) slot = CB; else if (di == 1 && dj == 0) slot = CH; else if (di == -1 && dj == 0) slot = CI;
            else if (di == 0 && dj == 1) slot = CL; else if (di == 0 && dj == -1) slot = CM;
        } else {
            if (di == 0 && dj == 0) slot = CC; else if (di == 1 && dj == 0) slot = CJ; else if (di == -1 && dj == 0) slot = CK;
            else if (di == 0 && dj == 1) slot = CN; else if (di == 0 && dj == -1) slot = CO;
        }
        if (slot >= 0) coef[(long long)slot * d.npad + kidx(d, i, k, j)] = tv;
        else leak = fabsf(tv);
    }
    // max |T| off the stencil; non-negative floats order like their bit patterns
    for (int o = 16; o > 0; o >>= 1) leak = fmaxf(leak, __shfl_xor_sync(0xffffffffu, leak, o));
    if ((threadIdx.x & 31) == 0 && leak > 0.0f) atomicMax(max_leak_bits, __float_as_uint(leak));
}

void launch_probe_record(const Dims &d, const float *T, float *coef, int ca, int cb, int cc, unsigned int *leak,
                         cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.nz, d.ny);
    probe_record_kernel<<<g, b, 0, st>>>(d, T, coef, ca, cb, cc, leak);
    count_launch(1);
}

// ---------------------------------------------------------------------------
// init_module_vars (:2274-2421): dz_if, dzdx_surf, dzdy_surf, adv_dz_col.
// ---------------------------------------------------------------------------
__global__ void module_vars_kernel(Dims d, const float *__restrict__ adz, const float *__restrict__ dzdx,
                                   const float *__restrict__ dzdy, const float *__restrict__ nterr, float *dz_if,
                                   float *dzdx_surf, float *dzdy_surf, float *adz_col)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx) return;
    const int nz = d.nz;
    for (int k = 2; k <= nz; k++)
        dz_if[zidx(d, i, k, j)] = (adz[cidx(d, i, k, j)] + adz[cidx(d, i, k - 1, j)]) / 2.0f;
    dz_if[zidx(d, i, 1, j)] = adz[cidx(d, i, 1, j)];
    dz_if[zidx(d, i, nz + 1, j)] = adz[cidx(d, i, nz, j)];
    float sx = dzdx[cidx(d, i, 1, j)], sy = dzdy[cidx(d, i, 1, j)];
    if (i >= 2 && i <= d.nx - 1) sx = (nterr[i2(d, i + 1, j)] - nterr[i2(d, i - 1, j)]) / (2.0f * d.dx);
    if (j >= 2 && j <= d.ny - 1) sy = (nterr[i2(d, i, j + 1)] - nterr[i2(d, i, j - 1)]) / (2.0f * d.dx);
    dzdx_surf[i2(d, i, j)] = sx;
    dzdy_surf[i2(d, i, j)] = sy;
    if (i == 1 && j == 1)
        for (int k = 1; k <= nz; k++) adz_col[k - 1] = adz[cidx(d, 1, k, 1)];
}

void launch_module_vars(const Dims &d, const float *adz, const float *dzdx, const float *dzdy, const float *nterr,
                        float *dz_if, float *dzdx_surf, float *dzdy_surf, float *adz_col, cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.ny);
    module_vars_kernel<<<g, b, 0, st>>>(d, adz, dzdx, dzdy, nterr, dz_if, dzdx_surf, dzdy_surf, adz_col);
    count_launch(1);
}

// ---------------------------------------------------------------------------
// Analytic coefficients.  mode 0 = initialize_coefs + update_coefs_host (first
// call, :2424-2552); mode 1 = update_coefs_gpu (alpha refresh, :2555-2603),
// which rewrites A, B, C only.
// ---------------------------------------------------------------------------
__global__ void coefs_kernel(Dims d, Metrics m, const float *__restrict__ alpha, float *coef, int mode)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1, j = blockIdx.z + 1;
    if (i > d.nx) return;
    const int nz = d.nz;
    const float dx = d.dx;
    long long c = cidx(d, i, k, j);
    long long o = kidx(d, i, k, j);
    float *A = coef + (long long)CA * d.npad, *B = coef + (long long)CB * d.npad, *C = coef + (long long)CC * d.npad;
    float dzdx_k = m.dzdx[c], dzdy_k = m.dzdy[c], a_k = alpha[c];
    float X_num = -((m.dzdx_u[uidx(d, i + 1, k, j)] / m.ju[uidx(d, i + 1, k, j)] - m.dzdx_u[uidx(d, i, k, j)] / m.ju[uidx(d, i, k, j)]) +
                    (m.dzdy_v[cidx(d, i, k, j + 1)] / m.jv[cidx(d, i, k, j + 1)] - m.dzdy_v[cidx(d, i, k, j)] / m.jv[cidx(d, i, k, j)]));
    if (mode == 0) {
#define ADZ(kk) m.adz[cidx(d, 1, (kk), 1)]
        float inv = 1.0f / (dx * dx);
        float md = 2.0f * dx * (m.dz_if[zidx(d, 1, k + 1, 1)] + m.dz_if[zidx(d, 1, k, 1)]);
        float gx = dzdx_k / m.jac[c], gy = dzdy_k / m.jac[c];
        float ux1 = m.dzdx_u[uidx(d, i + 1, k, j)] / m.ju[uidx(d, i + 1, k, j)];
        float ux0 = m.dzdx_u[uidx(d, i, k, j)] / m.ju[uidx(d, i, k, j)];
        float vy1 = m.dzdy_v[cidx(d, i, k, j + 1)] / m.jv[cidx(d, i, k, j + 1)];
        float vy0 = m.dzdy_v[cidx(d, i, k, j)] / m.jv[cidx(d, i, k, j)];
        coef[(long long)CD * d.npad + o] = inv;
        coef[(long long)CE * d.npad + o] = inv;
        coef[(long long)CF * d.npad + o] = inv;
        coef[(long long)CG * d.npad + o] = inv;
        coef[(long long)CH * d.npad + o] = -(gx + ux1) / md;
        coef[(long long)CI * d.npad + o] = (gx + ux0) / md;
        coef[(long long)CL * d.npad + o] = -(gy + vy1) / md;
        coef[(long long)CM * d.npad + o] = (gy + vy0) / md;
        coef[(long long)CJ * d.npad + o] = (gx + ux1) / md;
        coef[(long long)CK * d.npad + o] = -(gx + ux0) / md;
        coef[(long long)CN * d.npad + o] = (gy + vy1) / md;
        coef[(long long)CO * d.npad + o] = -(gy + vy0) / md;
        float M_up, M_dwn;
        if (k == 1) {
            long long cp = cidx(d, i, k + 1, j);
            float dzdx_p = m.dzdx[cp], dzdy_p = m.dzdy[cp], a_p = alpha[cp], jw = m.jw[c];
            M_up = dzdx_k * (dzdx_k * ADZ(k + 1) + dzdx_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
            M_dwn = dzdx_k * m.dzdx_surf[i2(d, i, j)];
            M_up = M_up + dzdy_k * (dzdy_k * ADZ(k + 1) + dzdy_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
            M_dwn = M_dwn + dzdy_k * m.dzdy_surf[i2(d, i, j)];
            M_up = M_up + (a_k * a_k * ADZ(k + 1) + a_p * a_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
            M_dwn = M_dwn + a_k * a_k;
        } else if (k == nz) {
            long long cm = cidx(d, i, k - 1, j);
            float dzdx_m = m.dzdx[cm], dzdy_m = m.dzdy[cm], a_m = alpha[cm], jwm = m.jw[cm];
            M_up = dzdx_k * (dzdx_k * ADZ(k) + dzdx_k * ADZ(k)) / (ADZ(k) + ADZ(k));
            M_dwn = dzdx_k * (dzdx_k * ADZ(k - 1) + dzdx_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
            M_up = M_up + dzdy_k * (dzdy_k * ADZ(k) + dzdy_k * ADZ(k)) / (ADZ(k) + ADZ(k));
            M_dwn = M_dwn + dzdy_k * (dzdy_k * ADZ(k - 1) + dzdy_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
            M_up = M_up + (a_k * a_k * ADZ(k) + a_k * a_k * ADZ(k)) / (ADZ(k) + ADZ(k));
            M_dwn = M_dwn + (a_k * a_k * ADZ(k - 1) + a_m * a_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
        } else {
            long long cp = cidx(d, i, k + 1, j), cm = cidx(d, i, k - 1, j);
            float dzdx_p = m.dzdx[cp], dzdy_p = m.dzdy[cp], a_p = alpha[cp], jw = m.jw[c];
            float dzdx_m = m.dzdx[cm], dzdy_m = m.dzdy[cm], a_m = alpha[cm], jwm = m.jw[cm];
            M_up = dzdx_k * (dzdx_k * ADZ(k + 1) + dzdx_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
            M_dwn = dzdx_k * (dzdx_k * ADZ(k - 1) + dzdx_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
            M_up = M_up + dzdy_k * (dzdy_k * ADZ(k + 1) + dzdy_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
            M_dwn = M_dwn + dzdy_k * (dzdy_k * ADZ(k - 1) + dzdy_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
            M_up = M_up + (a_k * a_k * ADZ(k + 1) + a_p * a_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
            M_dwn = M_dwn + (a_k * a_k * ADZ(k - 1) + a_m * a_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
        }
        float Bv = M_up / (m.jac[c] * ADZ(k) * m.dz_if[zidx(d, 1, k + 1, 1)]);
        float Cv = M_dwn / (m.jac[c] * ADZ(k) * m.dz_if[zidx(d, 1, k, 1)]);
        float Av = -4.0f / (dx * dx) - Bv - Cv;
        float mixed = (m.dz_if[zidx(d, i, k + 1, j)] + m.dz_if[zidx(d, i, k, j)]) * 2.0f * dx;
        float X = X_num / mixed;
        A[o] = Av;
        B[o] = Bv + X;
        C[o] = Cv - X;
#undef ADZ
    } else {
        float adz_k = m.adz_col[k - 1];
        float M_up, M_dwn;
        if (k == nz) {
            M_up = dzdx_k * dzdx_k + dzdy_k * dzdy_k + a_k * a_k;
        } else {
            float adz_p = m.adz_col[k], sum_up = adz_k + adz_p;
            long long cp = cidx(d, i, k + 1, j);
            float jw = m.jw[c];
            M_up = dzdx_k * (dzdx_k * adz_p + m.dzdx[cp] * adz_k) / sum_up / jw +
                   dzdy_k * (dzdy_k * adz_p + m.dzdy[cp] * adz_k) / sum_up / jw +
                   (a_k * a_k * adz_p + alpha[cp] * alpha[cp] * adz_k) / sum_up / jw;
        }
        if (k == 1) {
            M_dwn = dzdx_k * m.dzdx_surf[i2(d, i, j)] + dzdy_k * m.dzdy_surf[i2(d, i, j)] + a_k * a_k;
        } else {
            float adz_m = m.adz_col[k - 2], sum_dw = adz_k + adz_m;
            long long cm = cidx(d, i, k - 1, j);
            float jwm = m.jw[cm];
            M_dwn = dzdx_k * (dzdx_k * adz_m + m.dzdx[cm] * adz_k) / sum_dw / jwm +
                    dzdy_k * (dzdy_k * adz_m + m.dzdy[cm] * adz_k) / sum_dw / jwm +
                    (a_k * a_k * adz_m + alpha[cm] * alpha[cm] * adz_k) / sum_dw / jwm;
        }
        float Bv = M_up / (m.jac[c] * adz_k * m.dz_if[zidx(d, 1, k + 1, 1)]);
        float Cv = M_dwn / (m.jac[c] * adz_k * m.dz_if[zidx(d, 1, k, 1)]);
        float mixed = (m.dz_if[zidx(d, i, k + 1, j)] + m.dz_if[zidx(d, i, k, j)]) * 2.0f * dx;
        float X = X_num / mixed;
        Bv = Bv + X;
        Cv = Cv - X;
        B[o] = Bv;
        C[o] = Cv;
        A[o] = -4.0f / (dx * dx) - Bv - Cv;
    }
}

void launch_coefs(const Dims &d, const Metrics &m, const float *alpha, float *coef, int mode, cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.nz, d.ny);
    coefs_kernel<<<g, b, 0, st>>>(d, m, alpha, coef, mode);
    count_launch(1);
}

// Per-column FP64 data of the analytic bottom/top rows (spmv :950-988).
__global__ void bccol_kernel(Dims d, Metrics m, const float *__restrict__ alpha, BcCol *bc)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx) return;
    double two_dx = 2.0 * (double)d.dx;
    double dzdx_s = (double)m.dzdx_surf[i2(d, i, j)];
    double dzdy_s = (double)m.dzdy_surf[i2(d, i, j)];
    double dz_kp1 = (double)m.dz_if[zidx(d, i, 1, j)];
    double al = (double)alpha[cidx(d, i, 1, j)];
    double denom = 2.0 * (dzdx_s * dzdx_s + dzdy_s * dzdy_s + al * al) / (double)m.jac[cidx(d, i, 1, j)];
    BcCol b;
    b.cx = dzdx_s / (denom * two_dx);
    b.cy = dzdy_s / (denom * two_dx);
    b.m1 = -1.0 / dz_kp1;
    b.p1 = 1.0 / dz_kp1;
    b.dztop = (double)m.dz_if[zidx(d, i, d.nz + 1, j)];
    bc[(long long)j * d.mx + i] = b;
}

void launch_bccol(const Dims &d, const Metrics &m, const float *alpha, BcCol *bc, cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.ny);
    bccol_kernel<<<g, b, 0, st>>>(d, m, alpha, bc);
    count_launch(1);
}

// extract_diagonal (:1041-1075) over all rows; padding stays zero.
template <typename V>
__global__ void diag_kernel(Dims d, const float *__restrict__ coefA, const float *__restrict__ dz_if, V *Dinv, int probed)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int k = blockIdx.y, j = blockIdx.z;
    if (i >= d.mx) return;
    double dd;
    if (i <= 0 || j <= 0 || i >= d.mx - 1 || j >= d.my - 1) dd = 1.0;
    else if (k >= d.mz - 1) dd = probed ? 1.0 : 1.0 / (double)dz_if[zidx(d, i, k, j)];
    else if (k <= 0) dd = probed ? 1.0 : -1.0 / (double)dz_if[zidx(d, i, k + 1, j)];
    else dd = (double)coefA[kidx(d, i, k, j)];
    if (fabs(dd) < BREAKDOWN_EPS) dd = copysign(BREAKDOWN_EPS, dd);
    Dinv[kidx(d, i, k, j)] = (V)(1.0 / dd);
}

template <typename V>
void launch_diag(const Dims &d, const float *coefA, const float *dz_if, V *Dinv, int probed, cudaStream_t st)
{
    dim3 b(128), g((d.mx + 127) / 128, d.mz, d.my);
    diag_kernel<V><<<g, b, 0, st>>>(d, coefA, dz_if, Dinv, probed);
    count_launch(1);
}
template void launch_diag<double>(const Dims &, const float *, const float *, double *, int, cudaStream_t);
template void launch_diag<float>(const Dims &, const float *, const float *, float *, int, cudaStream_t);

// compute_rhs_3d (:1513-1530): b = real(-2*div, c_double) on interior rows, 0 elsewhere.
template <typename V>
__global__ void rhs_kernel(Dims d, const float *__restrict__ div, V *rhs)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int k = blockIdx.y, j = blockIdx.z;
    if (i >= d.mx) return;
    double b = 0.0;
    if (!(i <= 0 || j <= 0 || i >= d.mx - 1 || j >= d.my - 1 || k <= 0 || k >= d.mz - 1))
        b = (double)(-2.0f * div[cidx(d, i, k, j)]);
    rhs[kidx(d, i, k, j)] = (V)b;
}

template <typename V>
void launch_rhs(const Dims &d, const float *div, V *rhs, cudaStream_t st)
{
    dim3 b(128), g((d.mx + 127) / 128, d.mz, d.my);
    rhs_kernel<V><<<g, b, 0, st>>>(d, div, rhs);
    count_launch(1);
}
template void launch_rhs<double>(const Dims &, const float *, double *, cudaStream_t);
template void launch_rhs<float>(const Dims &, const float *, float *, cudaStream_t);

// NaN count of the input divergence and alpha min/max (:319-329, :411-421), one pass.
__global__ void scan_inputs_kernel(long long n, const float *__restrict__ div, const float *__restrict__ alpha,
                                   unsigned int *nan_count, unsigned int *amin_bits, unsigned int *amax_bits)
{
    unsigned int cnt = 0;
    float mn = 3.4e38f, mx = -3.4e38f;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        float dv = div[q];
        if (dv != dv) cnt++;
        float a = alpha[q];
        mn = fminf(mn, a);
        mx = fmaxf(mx, a);
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (cnt) atomicAdd(nan_count, cnt);
        // order-preserving map of floats to unsigned ints
        unsigned int bmn = __float_as_uint(mn), bmx = __float_as_uint(mx);
        bmn = (bmn & 0x80000000u) ? ~bmn : (bmn | 0x80000000u);
        bmx = (bmx & 0x80000000u) ? ~bmx : (bmx | 0x80000000u);
        atomicMin(amin_bits, bmn);
        atomicMax(amax_bits, bmx);
    }
}

void launch_scan_inputs(long long n, const float *div, const float *alpha, unsigned int *out3, cudaStream_t st)
{
    scan_inputs_kernel<<<296, 256, 0, st>>>(n, div, alpha, out3, out3 + 1, out3 + 2);
    count_launch(1);
}

}  // namespace hw

namespace hw {

// ---------------------------------------------------------------------------
// The steps either side of the solve in update_winds (wind.F90), caller layouts,
// 1-based indices, Fortran's left-to-right FP32 order (this unit: -fmad=false).
// ---------------------------------------------------------------------------
// calc_w_real (wind.F90:1175-1227) at cell (i, k, j); w_grid may be null (zero)
__device__ __forceinline__ float w_real_at(const Dims &d, const Metrics &m, const float *u, const float *v,
                                           const float *w_grid, int i, int k, int j)
{
    const long long c = cidx(d, i, k, j);
    float lo = 0.0f, hi = 0.0f;
    if (w_grid) {
        hi = w_grid[c] * m.jw[c];
        if (k > 1) lo = w_grid[cidx(d, i, k - 1, j)] * m.jw[cidx(d, i, k - 1, j)];
    }
    const long long u0 = uidx(d, i, k, j), u1 = uidx(d, i + 1, k, j);
    const long long v0 = cidx(d, i, k, j), v1 = cidx(d, i, k, j + 1);
    return (u[u0] * m.dzdx_u[u0] + u[u1] * m.dzdx_u[u1]) * 0.5f + (v[v0] * m.dzdy_v[v0] + v[v1] * m.dzdy_v[v1]) * 0.5f +
           (lo + hi) * 0.5f;
}

__global__ void w_real_kernel(Dims d, Metrics m, const float *__restrict__ u, const float *__restrict__ v,
                              const float *__restrict__ w_grid, float *__restrict__ w_real)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1;
    int j = blockIdx.z + 1;
    if (i > d.nx) return;
    w_real[cidx(d, i, k, j)] = w_real_at(d, m, u, v, w_grid, i, k, j);
}

// calc_idealized_wgrid (wind.F90:940-998): one thread per column
__global__ void idealized_wgrid_kernel(Dims d, Metrics m, const float *__restrict__ u, const float *__restrict__ v,
                                       const float *__restrict__ w_real_field, float *__restrict__ w)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx) return;
    float cur = w_real_field[cidx(d, i, 1, j)] - w_real_at(d, m, u, v, nullptr, i, 1, j);
    for (int k = 1; k <= d.nz - 1; k++) {
        const long long c = cidx(d, i, k, j), cp = cidx(d, i, k + 1, j);
        const float nxt = w_real_field[cp] - w_real_at(d, m, u, v, nullptr, i, k + 1, j);
        float wk = (cur * m.adz[cp] + nxt * m.adz[c]) / (m.adz[c] + m.adz[cp]);
        w[c] = wk / m.jw[c];
        cur = nxt;
    }
    w[cidx(d, i, d.nz, j)] = 0.0f;
}

// calc_w (wind.F90:201-248): upward integration of the horizontal divergence per column
__global__ void calc_w_kernel(Dims d, Metrics m, const float *__restrict__ div, const float *__restrict__ rho,
                              float *__restrict__ w, int adv_den)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > d.nx) return;
    const int nz = d.nz;
    float w_prev = 0.0f, rho_prev = 0.0f, jw_prev = 0.0f;
    for (int k = 1; k <= nz; k++) {
        const long long c = cidx(d, i, k, j);
        const float dz = m.adz[c], jw = m.jw[c], dv = div[c];
        float wk;
        if (adv_den) {
            float rho_i;
            if (k < nz) {
                const long long cp = cidx(d, i, k + 1, j);
                rho_i = (rho[c] * m.adz[cp] + rho[cp] * dz) / (dz + m.adz[cp]);
            } else rho_i = rho[c];
            if (k == 1) wk = 0.0f - dv * dz / (jw * rho_i);
            else wk = ((w_prev * rho_prev * jw_prev) - dv * dz) / (jw * rho_i);
            rho_prev = rho_i;
        } else {
            if (k == 1) wk = (0.0f - dv * dz) / (jw);
            else wk = (w_prev * jw_prev - dv * dz) / (jw);
        }
        w[c] = wk;
        w_prev = wk;
        jw_prev = jw;
    }
}

// update_stability (wind.F90:1421-1565) with calc_dry_stability, calc_Ri and
// calc_froude (atm_utilities.F90:466-546): one thread per column (i, j), all
// levels; FP32 in Fortran's order of operations.  The wind-direction sector
// comes from atan2f, which is not correctly rounded on either side: a cell
// whose direction lies within an ulp of a 5-degree sector edge can pick the
// neighbouring sector's blocking height.
constexpr float STAB_GRAVITY = 9.81f;          // mod_wrf_constants gravity
constexpr float STAB_RAD2DEG = 57.2957779371f; // wind.F90:39

__device__ __forceinline__ float dry_stability(float th_top, float th_bot, float z_top, float z_bot, bool has_surf,
                                               float th_surf)
{
    if (has_surf) return STAB_GRAVITY * (th_top - th_bot) / ((z_top - z_bot) * th_surf);
    return STAB_GRAVITY * (th_top - th_bot) / ((z_top - z_bot) * (th_top + th_bot) / 2.0f);
}

__global__ void update_stability_kernel(Dims d, const float *__restrict__ u, const float *__restrict__ v,
                                        const float *__restrict__ z, const float *__restrict__ theta,
                                        const float *__restrict__ fterr, int nsect, int froude_mode,
                                        float *__restrict__ froude, float *__restrict__ blk_ri)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1;
    if (i > d.nx) return;
    const long long ncell = (long long)d.nx * d.ny * d.nz;
    int rk = d.nz; // Ri_k_max (:1444-1454)
    for (int k = 2; k <= d.nz; k++)
        if (z[cidx(d, i, k, j)] - z[cidx(d, i, 1, j)] > 100.0f) {
            rk = max(2, k - 1);
            break;
        }
    const float us = (u[uidx(d, i, 5, j)] + u[uidx(d, i + 1, 5, j)]) / 2.0f; // u_shear(:, kms, :) (:1462-1465)
    const float vs = (v[cidx(d, i, 5, j)] + v[cidx(d, i, 5, j + 1)]) / 2.0f;
    const float th_b = theta[cidx(d, i, 1, j)], th_t = theta[cidx(d, i, rk, j)];
    const float z_b = z[cidx(d, i, 1, j)], z_t = z[cidx(d, i, rk, j)];
    // calc_Ri of the column's bulk stability (:1482-1495)
    const float stab = dry_stability(th_t, th_b, z_t, z_b, false, 0.0f);
    const float dz = z_t - z_b, a = us / dz, b = vs / dz;
    const float den = a * a + b * b;
    const float ri = den == 0.0f ? 10.0f : stab / den;
    for (int k = 1; k <= d.nz; k++) {
        const long long o = cidx(d, i, k, j);
        blk_ri[o] = k < d.nz ? ri : 10.0f;
        float fr = 0.1f;
        if (froude_mode && k < d.nz) { // (:1503-1560)
            const float um = (u[uidx(d, i, k, j)] + u[uidx(d, i + 1, k, j)]) / 2.0f;
            const float vm = (v[cidx(d, i, k, j)] + v[cidx(d, i, k, j + 1)]) / 2.0f;
            const float ws = sqrtf(um * um + vm * vm);
            float wd = atan2f(-um, -vm) * STAB_RAD2DEG;
            if (wd <= 0.0f) wd = wd + 360.0f;
            if (wd == 360.0f) wd = 0.0f;
            const int dir = max(min((int)(wd / 5.0f) + 1, nsect), 1);
            const float tf = fterr[o + (long long)(dir - 1) * ncell];
            const float st = dry_stability(theta[cidx(d, i, k + 1, j)], theta[o], z[cidx(d, i, k + 1, j)], z[o], true,
                                           th_b);
            const float bv = sqrtf(fmaxf(st, 0.0f));
            const float fden = tf * bv;
            fr = fden == 0.0f ? 100.0f : ws / fden;
        }
        froude[o] = fr;
    }
}

void launch_update_stability(const Dims &d, const float *u, const float *v, const float *z, const float *theta,
                             const float *fterr, int nsect, int froude_mode, float *froude, float *blk_ri,
                             cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.ny);
    update_stability_kernel<<<g, b, 0, st>>>(d, u, v, z, theta, fterr, nsect, froude_mode, froude, blk_ri);
    count_launch(1);
}

// calc_alpha (wind.F90:1102-1173), elementwise part; (1/Fr)**4 as (t*t)*(t*t)
__global__ void calc_alpha_kernel(Dims d, const float *__restrict__ froude, float *__restrict__ alpha)
{
    const long long n = (long long)d.nx * d.nz * d.ny;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const float t = 1.0f / froude[q];
        const float t2 = t * t;
        const float p = t2 * t2;
        const float mx = p > 0.00001f ? p : 0.00001f;
        float a = 1.0f - 0.5f * mx * (sqrtf(1.0f + 4.0f / mx) - 1.0f);
        a = sqrtf(a > 0.00001f ? a : 0.00001f);
        a = a > 0.2f ? a : 0.2f;
        a = a < 2.0f ? a : 2.0f;
        const int k = (int)((q / d.nx) % d.nz) + 1;
        alpha[q] = k == d.nz ? 0.2f : a;
    }
}

// one of the four boundary copies of calc_alpha: side 0 south (j <= h), 1 west
// (i <= h), 2 north (j > ny - h), 3 east (i > nx - h); whole columns
__global__ void alpha_edge_kernel(Dims d, float *__restrict__ alpha, int h, int side)
{
    const int ni = (side == 1 || side == 3) ? h : d.nx, nj = (side == 0 || side == 2) ? h : d.ny;
    const long long n = (long long)ni * nj * d.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int a = (int)(q % ni) + 1;
        long long r = q / ni;
        int k = (int)(r % d.nz) + 1, b = (int)(r / d.nz) + 1;
        int i = a, j = b, is = a, js = b;
        if (side == 0) js = h + 1;
        else if (side == 1) is = h + 1;
        else if (side == 2) { j = d.ny - h + b; js = d.ny - h; }
        else { i = d.nx - h + a; is = d.nx - h; }
        alpha[cidx(d, i, k, j)] = alpha[cidx(d, is, k, js)];
    }
}

// one pass of smooth_array_3d, ydim = 3 (array_utilities.F90:322-397): x-y box
// mean with clamped indices, double sum (y offset outer, x inner)
__global__ void smooth_xy_kernel(Dims d, const float *__restrict__ in, float *__restrict__ out, int w)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int k = blockIdx.y + 1;
    int j = blockIdx.z + 1;
    if (i > d.nx) return;
    double cur = 0.0;
    for (int dj = -w; dj <= w; dj++) {
        const int jj = j + dj < 1 ? 1 : (j + dj > d.ny ? d.ny : j + dj);
        for (int di = -w; di <= w; di++) {
            const int ii = i + di < 1 ? 1 : (i + di > d.nx ? d.nx : i + di);
            cur = cur + (double)in[cidx(d, ii, k, jj)];
        }
    }
    const int nc = 2 * w + 1;
    out[cidx(d, i, k, j)] = (float)(cur / (double)(nc * nc));
}

void launch_w_real(const Dims &d, const Metrics &m, const float *u, const float *v, const float *w_grid, float *w_real,
                   cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.nz, d.ny);
    w_real_kernel<<<g, b, 0, st>>>(d, m, u, v, w_grid, w_real);
    count_launch(1);
}

void launch_idealized_wgrid(const Dims &d, const Metrics &m, const float *u, const float *v, const float *w_real_field,
                            float *w, cudaStream_t st)
{
    dim3 b(64), g((d.nx + 63) / 64, d.ny);
    idealized_wgrid_kernel<<<g, b, 0, st>>>(d, m, u, v, w_real_field, w);
    count_launch(1);
}

void launch_calc_w(const Dims &d, const Metrics &m, const float *div, const float *rho, float *w, int adv_den,
                   cudaStream_t st)
{
    dim3 b(64), g((d.nx + 63) / 64, d.ny);
    calc_w_kernel<<<g, b, 0, st>>>(d, m, div, rho, w, adv_den);
    count_launch(1);
}

void launch_calc_alpha(const Dims &d, const float *froude, float *alpha, int halo, cudaStream_t st)
{
    const long long n = (long long)d.nx * d.nz * d.ny;
    calc_alpha_kernel<<<(int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16), 256, 0, st>>>(d, froude, alpha);
    count_launch(1);
    if (halo > 0)
        for (int side = 0; side < 4; side++) {
            alpha_edge_kernel<<<148, 256, 0, st>>>(d, alpha, halo, side);
            count_launch(1);
        }
}

void launch_smooth_xy(const Dims &d, const float *in, float *out, int w, cudaStream_t st)
{
    dim3 b(128), g((d.nx + 127) / 128, d.nz, d.ny);
    smooth_xy_kernel<<<g, b, 0, st>>>(d, in, out, w);
    count_launch(1);
}

}  // namespace hw
