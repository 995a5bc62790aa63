// kernels.h -- host-side launchers of the device kernels (internal interface).
#pragma once
#include "common.cuh"

namespace hw {

void count_launch(int n);

// Per-launch profiling hook: when a profiling pass is active (never during graph
// capture) each launcher brackets its kernel with CUDA events and records its
// name and algorithmic bytes (compulsory DRAM traffic of one launch).
struct ProfScope {
    ProfScope(const char *name, double bytes, cudaStream_t s);
    ~ProfScope();
    int slot;
    cudaStream_t s;
};

// k_model.cu
void launch_divergence(const Dims &d, const Metrics &m, const float *u, const float *v, const float *w,
                       const float *rho, float *div, int adv_den, int horz_only, int use_dqdt, cudaStream_t st);
template <typename V>
void launch_winds(const Dims &d, const Metrics &m, const V *x, const float *alpha, const float *rho, float *u, float *v,
                  float *w, int adv_den, cudaStream_t st);
template <typename V>
void launch_probe_pattern(const Dims &d, V *x, int ca, int cb, int cc, cudaStream_t st);
void launch_probe_record(const Dims &d, const float *T, float *coef, int ca, int cb, int cc, unsigned int *leak,
                         cudaStream_t st);
void launch_w_real(const Dims &d, const Metrics &m, const float *u, const float *v, const float *w_grid, float *w_real,
                   cudaStream_t st);
void launch_idealized_wgrid(const Dims &d, const Metrics &m, const float *u, const float *v, const float *w_real_field,
                            float *w, cudaStream_t st);
void launch_calc_w(const Dims &d, const Metrics &m, const float *div, const float *rho, float *w, int adv_den,
                   cudaStream_t st);
void launch_calc_alpha(const Dims &d, const float *froude, float *alpha, int halo, cudaStream_t st);
void launch_update_stability(const Dims &d, const float *u, const float *v, const float *z, const float *theta,
                             const float *fterr, int nsect, int froude_mode, float *froude, float *blk_ri,
                             cudaStream_t st);
void launch_smooth_xy(const Dims &d, const float *in, float *out, int w, cudaStream_t st);
void launch_module_vars(const Dims &d, const float *adz, const float *dzdx, const float *dzdy, const float *nterr,
                        float *dz_if, float *dzdx_surf, float *dzdy_surf, float *adz_col, cudaStream_t st);
void launch_coefs(const Dims &d, const Metrics &m, const float *alpha, float *coef, int mode, cudaStream_t st);
void launch_bccol(const Dims &d, const Metrics &m, const float *alpha, BcCol *bc, cudaStream_t st);
template <typename V>
void launch_diag(const Dims &d, const float *coefA, const float *dz_if, V *Dinv, int probed, cudaStream_t st);
template <typename V>
void launch_rhs(const Dims &d, const float *div, V *rhs, cudaStream_t st);
void launch_scan_inputs(long long n, const float *div, const float *alpha, unsigned int *out3, cudaStream_t st);

// k_krylov.cu -- operator, preconditioner and BiCGStab steps (generic schedule).
struct OpCtx {
    Dims d;
    const float *coef; // 15 * d.npad
    const BcCol *bc;   // mx * my
    int probed;
    int kc = 0;        // levels per work item of the float4 column-marching kernels (0: the default)
    int edges = 0;     // rank-edge sides of a decomposed subdomain (EDGE_* bits; 0: one rank)
};

struct RedBuf {
    double *partials; // >= red_blocks * 8
    int blocks;       // grid size of the reduction kernels
};

template <typename V>
void launch_spmv(const OpCtx &c, const V *x, V *y, const SolveState *gate, cudaStream_t st);
template <typename V>
void launch_precond_scale(const Dims &d, const V *in, V *out, const V *Dinv, SolveState *gate, int set_halt,
                          cudaStream_t st);
template <typename V>
void launch_s_precond(const Dims &d, const V *r, const V *v, V *s, V *shat, const V *Dinv, SolveState *stt,
                      cudaStream_t st);
template <typename V>
void launch_rich(const Dims &d, const V *in, V *out, const V *pres, const V *Dinv, const SolveState *gate,
                 cudaStream_t st);
template <typename V, typename X>
void launch_setup(const OpCtx &c, const X *x, const V *rhs, V *r, V *rhat, V *p, SolveState *stt, double *hist,
                  const RedBuf &rb, int restart, cudaStream_t st);
template <typename V>
void launch_spmv_sigma(const OpCtx &c, const V *phat, V *v, const V *rhat, SolveState *stt, const RedBuf &rb,
                       cudaStream_t st);
template <typename V>
void launch_spmv_dot5(const OpCtx &c, const V *shat, V *t, const V *s, const V *rhat, SolveState *stt, double *hist,
                      const RedBuf &rb, cudaStream_t st);
template <typename V, typename X>
void launch_update_xrp(const Dims &d, X *x, const V *phat, const V *shat, V *r, const V *s, const V *t, V *p,
                       const V *v, const SolveState *stt, cudaStream_t st);
void launch_state_reset(SolveState *stt, double tol_rel, double tol_abs, int max_iters, int stall_k, cudaStream_t st);
void launch_iteration_begin(SolveState *stt, cudaStream_t st);
// decomposed solve: apply the scalar step of kind 0 (set-up), 1 (sigma) or 2 (five dots) to global totals
void launch_dist_apply(SolveState *stt, double *hist, int kind, const double *tot, cudaStream_t st);
// zero a vector on the halo cells of the rank-edge sides (edges bits)
template <typename V>
void launch_zero_rank_edges(const Dims &d, int edges, V *x, cudaStream_t st);
// pack (unpack = 0) the owned boundary face next to `side` (0 W, 1 E, 2 S, 3 N) into buf, or
// unpack (unpack = 1) buf into the halo face of that side; FP64, (nz+2)(ny+2) or (nz+2)(nx+2) values
void launch_face(const Dims &d, double *x, int side, double *buf, int unpack, cudaStream_t st);
template <typename V, typename X>
void launch_true_residual(const OpCtx &c, const X *x, const V *rhs, V *r_out, const V *rhat, SolveState *stt,
                          int mode, const RedBuf &rb, cudaStream_t st);
template <typename A, typename B>
void launch_convert(long long n, const A *in, B *out, cudaStream_t st);

}  // namespace hw
