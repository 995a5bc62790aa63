// common.cuh -- layout, device state and small helpers shared by the kernels.
//
// HBM layout of every Krylov vector and of the 15 coefficient arrays: the
// reference's (0:nx+1, 0:nz+1, 0:ny+1) array (i fastest, then k, then j;
// wind_iterative.F90:101-103,359-370) with each i-row padded to a pitch P that
// is a multiple of 8 elements, and element i = 0 of a row stored at offset XO = 7,
// so the first physical cell i = 1 starts on a 32-byte sector.  Padding
// elements are zero in every vector and stay zero (every kernel writes real rows
// only, or writes values that are zero when their inputs are zero).
// Coefficients use the same indexing; only interior rows (1..nx, 1..nz, 1..ny)
// hold meaningful values.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hw {

constexpr int XO = 7;
constexpr int NCOEF = 15;
enum { CA = 0, CB, CC, CD, CE, CF, CG, CH, CI, CJ, CK, CL, CM, CN, CO };

struct Dims {
    int nx, ny, nz;
    int mx, my, mz;  // nx+2, ny+2, nz+2
    int P;           // row pitch (elements)
    long long plane; // P * mz
    long long npad;  // plane * my (elements per padded vector)
    float dx;
};

__host__ __device__ __forceinline__ long long kidx(const Dims &d, int i, int k, int j)
{
    return ((long long)j * d.mz + k) * d.P + i + XO;
}
// Caller (Fortran) layouts, 1-based indices.
__host__ __device__ __forceinline__ long long cidx(const Dims &d, int i, int k, int j)
{
    return (long long)(i - 1) + (long long)d.nx * ((long long)(k - 1) + (long long)d.nz * (j - 1));
}
__host__ __device__ __forceinline__ long long uidx(const Dims &d, int i, int k, int j)
{
    return (long long)(i - 1) + (long long)(d.nx + 1) * ((long long)(k - 1) + (long long)d.nz * (j - 1));
}
__host__ __device__ __forceinline__ long long zidx(const Dims &d, int i, int k, int j)
{
    return (long long)(i - 1) + (long long)d.nx * ((long long)(k - 1) + (long long)(d.nz + 1) * (j - 1));
}
__host__ __device__ __forceinline__ long long i2(const Dims &d, int i, int j) { return (long long)(i - 1) + (long long)d.nx * (j - 1); }
__host__ __device__ __forceinline__ long long i2u(const Dims &d, int i, int j) { return (long long)(i - 1) + (long long)(d.nx + 1) * (j - 1); }

// Metric fields on the device, caller layout (copied once at init).
struct Metrics {
    const float *jac, *ju, *jv, *jw, *dzdx, *dzdy, *dzdx_u, *dzdy_v, *adz, *nterr;
    const float *mf_mx_u, *mf_my_v, *mf_my_u, *mf_mx_v, *mf_mxy;
    const float *dz_if, *dzdx_surf, *dzdy_surf, *adz_col;
};

// Per-column data of the analytic boundary rows (spmv :950-988), FP64.
struct BcCol {
    double cx, cy, m1, p1, dztop;
};

// Device-resident BiCGStab state: the scalars of bicgstab_solve (:563-570) plus
// the control flags that replace the host-side `exit` statements.
struct SolveState {
    double rho, alpha, omega, beta, sigma;
    double rnorm, res0, bnorm2, target;
    double tol_rel, tol_abs;
    double true_res;
    int it;         // current iteration number (n_iters_out)
    int max_iters;
    int status;     // 0 converged, 1 iteration cap, 2 breakdown
    int stop;       // no further Krylov work this solve
    int halt;       // no further x updates this solve
    int upd_r;      // update_xrp: also form the new r
    int upd_p;      // update_xrp: also form the new p
    int replacements;
    unsigned int ticket[8];
    int err;        // device-side error flag (bounded waits)
    int profile;    // profiling pass: kernels ignore the stop/halt flags
    int stall_k;    // stall detector window (0 = off)
    int best_it;    // iteration of the best recurrence norm so far
    double best_rn; // best recurrence norm so far
    int dist;       // decomposed solve: reductions publish their local totals in dist_tot and the
                    // host applies the scalar steps to the totals summed over all ranks
    double dist_tot[5];
    double mr_theta; // composite learned preconditioner: the minimal-residual step along the U-Net's correction
};

// Rank-edge sides of a decomposed subdomain (bit mask): their ring cells are
// halo cells filled by the neighbouring rank, not rows of this rank's system.
enum { EDGE_W = 1, EDGE_E = 2, EDGE_S = 4, EDGE_N = 8 };
__host__ __device__ __forceinline__ bool owned_row(const Dims &d, int edges, int i, int j)
{
    return !((i == 0 && (edges & EDGE_W)) || (i == d.mx - 1 && (edges & EDGE_E)) || (j == 0 && (edges & EDGE_S)) ||
             (j == d.my - 1 && (edges & EDGE_N)));
}

constexpr double BREAKDOWN_EPS = 1.0e-30; // wind_iterative.F90:61

// Every C entry point starts here: it clears an error that an earlier CUDA call
// of the calling thread left pending (the host program's own, or another
// library's), so that the entry point's launch checks report its own errors
// only.  An error that breaks the context comes back from the next call that
// touches the device.
inline void api_entry() { (void)cudaGetLastError(); }

}  // namespace hw
