// capi.cu -- the C ABI of include/hicarw.h: per-nest handle, control flow of
// calc_iter_winds (wind_iterative.F90:295-532), probing (:1096-1248,
// wind.F90:1010-1099) and the device-driven BiCGStab loop.
//
// The loop: one CUDA graph holds `check_every` BiCGStab iterations (the kernel
// schedule of k_krylov.cu).  The host
// replays it and, one graph behind, reads the device-side `stop` flag through
// pinned memory, so the GPU never waits for the host inside a solve.  Kernels
// of an ended solve return immediately.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <map>
#include <algorithm>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/hicarw.h"
#include "common.cuh"
#include "kernels.h"
#include "mg.h"
#include "fgmres.h"
#include "unet.h"
#include "krylov_dev.cuh"

using namespace hw;

namespace hw {
static std::atomic<long long> g_launches{0};
static thread_local int g_capturing = 0;
static thread_local int g_capture_nodes = 0;
void count_launch(int n)
{
    if (g_capturing) g_capture_nodes += n;
    else g_launches += n;
}

struct ProfRec {
    std::string name; // copied: callers may pass a temporary buffer
    double bytes;
    cudaEvent_t a, b;
};
static thread_local int g_prof_on = 0;
static thread_local std::vector<ProfRec> g_prof;

ProfScope::ProfScope(const char *name, double bytes, cudaStream_t st) : slot(-1), s(st)
{
    if (!g_prof_on || g_capturing) return;
    ProfRec r{name, bytes, nullptr, nullptr};
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    cudaEventRecord(r.a, s);
    g_prof.push_back(r);
    slot = (int)g_prof.size() - 1;
}
ProfScope::~ProfScope()
{
    if (slot >= 0) cudaEventRecord(g_prof[slot].b, s);
}
}  // namespace hw

#define CK(call)                                                                                                       \
    do {                                                                                                               \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess) {                                                                                       \
            set_err(h, #call, e_);                                                                                     \
            return HICARW_ERR_CUDA;                                                                                    \
        }                                                                                                              \
    } while (0)

static thread_local std::string g_err_noh;

struct GraphKey {
    int prec, sweeps, chunk, solver, replace, precond;
    bool operator<(const GraphKey &o) const
    {
        if (precond != o.precond) return precond < o.precond;
        if (prec != o.prec) return prec < o.prec;
        if (sweeps != o.sweeps) return sweeps < o.sweeps;
        if (chunk != o.chunk) return chunk < o.chunk;
        if (solver != o.solver) return solver < o.solver;
        return replace < o.replace;
    }
};
struct GraphRec {
    cudaGraphExec_t exec;
    int nodes;
};

enum { V_X = 0, V_R, V_RHAT, V_P, V_PHAT, V_V, V_S, V_SHAT, V_T, V_RHS, V_DINV, V_PRES, NVEC };

struct hicarw_handle {
    Dims d;
    hicarw_options opt;
    int nest = 1;
    cudaStream_t cap = nullptr;
    // metric fields, caller layout
    float *mjac = nullptr, *mju = nullptr, *mjv = nullptr, *mjw = nullptr, *mdzdx = nullptr, *mdzdy = nullptr,
          *mdzdx_u = nullptr, *mdzdy_v = nullptr, *madz = nullptr, *mnterr = nullptr;
    float *mf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    float *dz_if = nullptr, *dzdx_surf = nullptr, *dzdy_surf = nullptr, *adz_col = nullptr;
    float *alpha = nullptr, *div = nullptr;
    float *coef = nullptr;
    BcCol *bc = nullptr;
    int vprec = -1; // precision of the allocated Krylov vectors
    void *vec[NVEC] = {};
    SolveState *st = nullptr;
    SolveState *hst = nullptr; // pinned host mirror
    int *hflag = nullptr;      // pinned stop flags (2 slots)
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    double *hist = nullptr;
    int hist_cap = 0;
    double *partials = nullptr;
    int red_blocks = 0;
    unsigned int *scan = nullptr; // nan count, alpha min, alpha max, probe leak
    unsigned int *hscan = nullptr;
    // staging for host pointers
    float *su = nullptr, *sv = nullptr, *sw = nullptr, *sT = nullptr, *srho = nullptr, *sdiv = nullptr;
    float *sprobe_u = nullptr, *sprobe_v = nullptr, *sprobe_w = nullptr;
    float *swork = nullptr; // cell-sized scratch of balance_uvw (divergence) and smooth_alpha (ping-pong)
    int structure_uploaded = 0, operator_probed = 0, precond_n_sweeps = 2;
    std::map<GraphKey, GraphRec> graphs;
    Mg mg;
    GmresState *gst = nullptr;      // FGMRES device state
    GmresState *fg_host = nullptr;  // pinned copy of its scalar head
    struct {
        hicarw_handle *h;
        int sweeps;
    } fg_pc;                        // preconditioner context of the FGMRES launches
    double *fgV = nullptr, *fgZ = nullptr, *fgW = nullptr;
    int fg_m = 0;
    int mg_dirty = 1;     // coefficients changed since the multigrid hierarchy was built
    hicarw_unet *unet = nullptr; // learned preconditioner (not owned)
    int unet_dirty = 1;   // coefficients changed since the network's operator features were computed
    int use_learned = 0;  // the current solve applies the learned preconditioner
    int use_mglearned = 0; // ... the V-cycle followed by the learned correction of its residual
    int tune_kc = 0;       // levels per work item of the float4 marching operator kernels (0: default)
    int edges = 0;         // decomposed solve: rank-edge sides of this subdomain (EDGE_* bits)
    double *dist_buf = nullptr; // decomposed solve: device staging of host-side totals (5 values)
    int tune_mg_feed = -1; // multigrid post-smoother feed: 1 tensor copies, 0 register-fed, -1 the build's choice
    int use_mg = 0;       // preconditioner of the solve being enqueued
    std::string err;
    long long launches_at_call = 0;
};

static void set_err(hicarw_handle *h, const char *what, cudaError_t e)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    if (h) h->err = buf;
    else g_err_noh = buf;
}

static const int BASE_PREC_SWEEPS = 2; // wind_iterative.F90:75
static const int MAX_PREC_SWEEPS = 4;  // wind_iterative.F90:76

extern "C" void hicarw_default_options(hicarw_options *o)
{
    memset(o, 0, sizeof(*o));
    o->max_iters = 1500;
    o->verbose = 0;
    o->tol_rel = 1.0e-5;
    o->tol_abs = 1.0e-10;
    o->krylov_precision = HICARW_KRYLOV_F64;
    o->solver = HICARW_SOLVER_REFERENCE;
    o->criterion = HICARW_CRIT_RECURRENCE;
    o->replace_every = 50;
    o->check_every = 8;
    o->precond = HICARW_PRECOND_JACOBI;
    o->stall_iters = 0;
    o->mg_omega = 0.8f;
    o->fgmres_restart = 30;
    o->mg_coarse_scale = 1.35f; // over-correction of the aggregation coarse grid: 35 -> 25 iterations at 512x512x48
    o->mg_skip_fine_presmooth = 0;
    o->mg_w_levels = 0;
    o->mg_precision = 0;
}

// V-cycle parameters from the options (read when its launches are enqueued).
static void mg_params(hicarw_handle *h)
{
    h->mg.omega = h->opt.mg_omega > 0.0f ? h->opt.mg_omega : 0.8f;
    h->mg.cscale = h->opt.mg_coarse_scale > 0.0f ? h->opt.mg_coarse_scale : 1.35f;
    h->mg.pre0 = h->opt.mg_skip_fine_presmooth ? 0 : 1;
    h->mg.wmask = h->opt.mg_w_levels & ~1;
    const int bf16 = h->opt.mg_precision == 1;
    if (bf16 != h->mg.bf16) h->mg_dirty = 1; // the finest level's factors and BF16 copy change
    h->mg.bf16 = bf16;
}

// The V-cycle of the handle's probed operator, with the tuned post-smoother feed.
static int mg_build_tuned(hicarw_handle *h, cudaStream_t s)
{
    if (mg_build(h->mg, h->d, h->coef, s) != 0) return -1;
    if (h->tune_mg_feed >= 0) h->mg.use_tma = h->tune_mg_feed ? 2 : 0;
    return 0;
}

static Metrics metrics_of(const hicarw_handle *h)
{
    Metrics m;
    m.jac = h->mjac; m.ju = h->mju; m.jv = h->mjv; m.jw = h->mjw; m.dzdx = h->mdzdx; m.dzdy = h->mdzdy;
    m.dzdx_u = h->mdzdx_u; m.dzdy_v = h->mdzdy_v; m.adz = h->madz; m.nterr = h->mnterr;
    m.mf_mx_u = h->mf[0]; m.mf_my_v = h->mf[1]; m.mf_my_u = h->mf[2]; m.mf_mx_v = h->mf[3]; m.mf_mxy = h->mf[4];
    m.dz_if = h->dz_if; m.dzdx_surf = h->dzdx_surf; m.dzdy_surf = h->dzdy_surf; m.adz_col = h->adz_col;
    return m;
}

static OpCtx opctx(const hicarw_handle *h)
{
    OpCtx c;
    c.d = h->d;
    c.coef = h->coef;
    c.bc = h->bc;
    c.probed = h->operator_probed;
    c.kc = h->tune_kc;
    c.edges = h->edges;
    return c;
}

static size_t n_cell(const Dims &d) { return (size_t)d.nx * d.nz * d.ny; }
static size_t n_u(const Dims &d) { return (size_t)(d.nx + 1) * d.nz * d.ny; }
static size_t n_v(const Dims &d) { return (size_t)d.nx * d.nz * (d.ny + 1); }

static cudaError_t dalloc(void **p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    return e;
}

static int ensure_vectors(hicarw_handle *h, int prec)
{
    const Dims &d = h->d;
    if (h->vprec == prec) return 0;
    // FP64 vectors for HICARW_KRYLOV_F64; FP32 otherwise, except lambda (V_X),
    // which HICARW_KRYLOV_F32_X64 accumulates in FP64
    const bool x_was64 = h->vprec == HICARW_KRYLOV_F64 || h->vprec == HICARW_KRYLOV_F32_X64;
    const bool x_is64 = prec == HICARW_KRYLOV_F64 || prec == HICARW_KRYLOV_F32_X64;
    void *nv[NVEC] = {};
    for (int q = 0; q < NVEC; q++) {
        const size_t es = prec == HICARW_KRYLOV_F64 || (q == V_X && x_is64) ? 8 : 4;
        CK(dalloc(&nv[q], (size_t)d.npad * es));
    }
    if (h->vprec >= 0) { // carry the warm-start lambda across a precision change
        if (x_is64 && !x_was64) launch_convert<float, double>(d.npad, (const float *)h->vec[V_X], (double *)nv[V_X], 0);
        else if (!x_is64 && x_was64) launch_convert<double, float>(d.npad, (const double *)h->vec[V_X], (float *)nv[V_X], 0);
        else CK(cudaMemcpy(nv[V_X], h->vec[V_X], (size_t)d.npad * (x_is64 ? 8 : 4), cudaMemcpyDeviceToDevice));
        CK(cudaDeviceSynchronize());
        for (int q = 0; q < NVEC; q++) cudaFree(h->vec[q]);
    }
    for (int q = 0; q < NVEC; q++) h->vec[q] = nv[q];
    h->vprec = prec;
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
    h->graphs.clear();
    return 0;
}

template <typename T>
static T *V(hicarw_handle *h, int q) { return (T *)h->vec[q]; }

// Krylov vector precision of the configured solve: the reference schedule takes
// the option, FGMRES is FP64.
static int solve_precision(const hicarw_handle *h)
{
    if (h->opt.solver == HICARW_SOLVER_REFERENCE) return h->opt.krylov_precision;
    return HICARW_KRYLOV_F64;
}

// Stage a caller array to the device when it lives in host memory.
static int stage_in(hicarw_handle *h, const float *src, float **buf, size_t n, int mem_kind, cudaStream_t s,
                    const float **out)
{
    if (mem_kind == HICARW_MEM_DEVICE || src == nullptr) { *out = src; return 0; }
    if (!*buf) CK(cudaMalloc((void **)buf, n * sizeof(float)));
    CK(cudaMemcpyAsync(*buf, src, n * sizeof(float), cudaMemcpyHostToDevice, s));
    *out = *buf;
    return 0;
}

// Options as the solve uses them.  HICARW_SOLVER_MIXED names the reference
// schedule with FP32 Krylov vectors, FP64 reductions and FP64 lambda, periodic
// FP64 residual replacement and the FP64 true-residual stop; the fused FP32
// schedule (HICARW_SOLVER_FUSED) and FP32 lambda (HICARW_KRYLOV_F32) no longer
// exist.
static int normalize_options(hicarw_options *o)
{
    if (o->krylov_precision != HICARW_KRYLOV_F64 && o->krylov_precision != HICARW_KRYLOV_F32_X64) return HICARW_ERR_ARG;
    if (o->solver == HICARW_SOLVER_FUSED) return HICARW_ERR_ARG;
    if (o->solver == HICARW_SOLVER_MIXED) {
        o->solver = HICARW_SOLVER_REFERENCE;
        o->krylov_precision = HICARW_KRYLOV_F32_X64;
        o->criterion = HICARW_CRIT_TRUE;
    }
    if (o->solver != HICARW_SOLVER_REFERENCE && o->solver != HICARW_SOLVER_FGMRES) return HICARW_ERR_ARG;
    if (o->mg_precision < 0 || o->mg_precision > 1) return HICARW_ERR_ARG;
    if (o->check_every <= 0) o->check_every = 8;
    if (o->replace_every <= 0) o->replace_every = 50;
    return 0;
}

extern "C" int hicarw_init_iter_winds(const hicarw_grid *g, const hicarw_options *opt, const hicarw_metrics *m,
                                      int mem_kind, void *stream, hicarw_handle **out)
{
    api_entry();
    if (!g || !m || !out || g->nx < 3 || g->ny < 3 || g->nz < 2 || !(g->dx > 0.0f)) return HICARW_ERR_ARG;
    hicarw_options o0;
    if (opt) o0 = *opt;
    else hicarw_default_options(&o0);
    if (normalize_options(&o0) != 0) return HICARW_ERR_ARG;
    hicarw_handle *h = new hicarw_handle();
    Dims &d = h->d;
    d.nx = g->nx; d.ny = g->ny; d.nz = g->nz;
    d.mx = d.nx + 2; d.my = d.ny + 2; d.mz = d.nz + 2;
    d.P = ((d.nx + 1 + XO + 1) + 7) / 8 * 8;
    d.plane = (long long)d.P * d.mz;
    d.npad = d.plane * d.my;
    d.dx = g->dx;
    h->nest = g->nest;
    h->opt = o0;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = 0;
#define ALLOC(p, n) do { cudaError_t e_ = dalloc((void **)&(p), (n)); if (e_ != cudaSuccess) { set_err(h, "cudaMalloc", e_); hicarw_finalize_iter_winds(h); return HICARW_ERR_CUDA; } } while (0)
    ALLOC(h->mjac, n_cell(d) * 4); ALLOC(h->mju, n_u(d) * 4); ALLOC(h->mjv, n_v(d) * 4); ALLOC(h->mjw, n_cell(d) * 4);
    ALLOC(h->mdzdx, n_cell(d) * 4); ALLOC(h->mdzdy, n_cell(d) * 4); ALLOC(h->mdzdx_u, n_u(d) * 4);
    ALLOC(h->mdzdy_v, n_v(d) * 4); ALLOC(h->madz, n_cell(d) * 4); ALLOC(h->mnterr, (size_t)d.nx * d.ny * 4);
    ALLOC(h->mf[0], (size_t)(d.nx + 1) * d.ny * 4); ALLOC(h->mf[1], (size_t)d.nx * (d.ny + 1) * 4);
    ALLOC(h->mf[2], (size_t)(d.nx + 1) * d.ny * 4); ALLOC(h->mf[3], (size_t)d.nx * (d.ny + 1) * 4);
    ALLOC(h->mf[4], (size_t)d.nx * d.ny * 4);
    ALLOC(h->dz_if, (size_t)d.nx * (d.nz + 1) * d.ny * 4); ALLOC(h->dzdx_surf, (size_t)d.nx * d.ny * 4);
    ALLOC(h->dzdy_surf, (size_t)d.nx * d.ny * 4); ALLOC(h->adz_col, (size_t)d.nz * 4);
    ALLOC(h->alpha, n_cell(d) * 4); ALLOC(h->div, n_cell(d) * 4);
    ALLOC(h->coef, (size_t)NCOEF * d.npad * 4);
    ALLOC(h->bc, (size_t)d.mx * d.my * sizeof(BcCol));
    ALLOC(h->st, sizeof(SolveState));
    h->red_blocks = 148 * 16;
    ALLOC(h->partials, (size_t)h->red_blocks * 8 * sizeof(double));
    ALLOC(h->scan, 8 * sizeof(unsigned int));
    h->hist_cap = h->opt.max_iters + 2;
    ALLOC(h->hist, (size_t)h->hist_cap * sizeof(double));
#undef ALLOC
    if (cudaMallocHost((void **)&h->hst, sizeof(SolveState)) != cudaSuccess ||
        cudaMallocHost((void **)&h->hflag, 4 * sizeof(int)) != cudaSuccess ||
        cudaMallocHost((void **)&h->hscan, 8 * sizeof(unsigned int)) != cudaSuccess) {
        hicarw_finalize_iter_winds(h);
        return HICARW_ERR_CUDA;
    }
    cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&h->ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&h->ev[1], cudaEventDisableTiming);
    cudaEventCreate(&h->t0);
    cudaEventCreate(&h->t1);
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    struct { float *dst; const float *src; size_t n; } cp[] = {
        {h->mjac, m->jacobian, n_cell(d)}, {h->mju, m->jacobian_u, n_u(d)}, {h->mjv, m->jacobian_v, n_v(d)},
        {h->mjw, m->jacobian_w, n_cell(d)}, {h->mdzdx, m->dzdx, n_cell(d)}, {h->mdzdy, m->dzdy, n_cell(d)},
        {h->mdzdx_u, m->dzdx_u, n_u(d)}, {h->mdzdy_v, m->dzdy_v, n_v(d)}, {h->madz, m->advection_dz, n_cell(d)},
        {h->mnterr, m->neighbor_terrain, (size_t)d.nx * d.ny},
        {h->mf[0], m->mapfac_mx_u, (size_t)(d.nx + 1) * d.ny}, {h->mf[1], m->mapfac_my_v, (size_t)d.nx * (d.ny + 1)},
        {h->mf[2], m->mapfac_my_u, (size_t)(d.nx + 1) * d.ny}, {h->mf[3], m->mapfac_mx_v, (size_t)d.nx * (d.ny + 1)},
        {h->mf[4], m->mapfac_mxy, (size_t)d.nx * d.ny}};
    for (auto &c : cp) {
        if (!c.src) { h->err = "missing metric field"; hicarw_finalize_iter_winds(h); return HICARW_ERR_ARG; }
        cudaError_t e = cudaMemcpyAsync(c.dst, c.src, c.n * sizeof(float), kind, s);
        if (e != cudaSuccess) { set_err(h, "metric copy", e); hicarw_finalize_iter_winds(h); return HICARW_ERR_CUDA; }
    }
    launch_module_vars(d, h->madz, h->mdzdx, h->mdzdy, h->mnterr, h->dz_if, h->dzdx_surf, h->dzdy_surf, h->adz_col, s);
    if ((rc = ensure_vectors(h, h->opt.krylov_precision)) != 0) { hicarw_finalize_iter_winds(h); return rc; }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_err(h, "init", e); hicarw_finalize_iter_winds(h); return HICARW_ERR_CUDA; }
    *out = h;
    return HICARW_OK;
}

extern "C" int hicarw_finalize_iter_winds(hicarw_handle *h)
{
    api_entry();
    if (!h) return HICARW_ERR_ARG;
    cudaDeviceSynchronize();
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
    h->graphs.clear();
    mg_free(h->mg);
    if (h->gst) cudaFree(h->gst);
    if (h->fg_host) cudaFreeHost(h->fg_host);
    if (h->fgV) cudaFree(h->fgV);
    if (h->fgZ) cudaFree(h->fgZ);
    if (h->fgW) cudaFree(h->fgW);
    void *ptrs[] = {h->mjac, h->mju, h->mjv, h->mjw, h->mdzdx, h->mdzdy, h->mdzdx_u, h->mdzdy_v, h->madz, h->mnterr,
                    h->mf[0], h->mf[1], h->mf[2], h->mf[3], h->mf[4], h->dz_if, h->dzdx_surf, h->dzdy_surf, h->adz_col,
                    h->alpha, h->div, h->coef, h->bc, h->st, h->hist, h->partials, h->scan, h->su, h->sv, h->sw,
                    h->sT, h->srho, h->sdiv, h->sprobe_u, h->sprobe_v, h->sprobe_w, h->swork};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int q = 0; q < NVEC; q++)
        if (h->vec[q]) cudaFree(h->vec[q]);
    if (h->hst) cudaFreeHost(h->hst);
    if (h->hflag) cudaFreeHost(h->hflag);
    if (h->hscan) cudaFreeHost(h->hscan);
    for (int q = 0; q < 2; q++)
        if (h->ev[q]) cudaEventDestroy(h->ev[q]);
    if (h->dist_buf) cudaFree(h->dist_buf);
    if (h->t0) cudaEventDestroy(h->t0);
    if (h->t1) cudaEventDestroy(h->t1);
    if (h->cap) cudaStreamDestroy(h->cap);
    delete h;
    return HICARW_OK;
}

extern "C" int hicarw_set_options(hicarw_handle *h, const hicarw_options *opt)
{
    api_entry();
    if (!h || !opt) return HICARW_ERR_ARG;
    hicarw_options o = *opt;
    if (normalize_options(&o) != 0) return HICARW_ERR_ARG;
    h->opt = o;
    if (h->opt.max_iters + 2 > h->hist_cap) {
        cudaFree(h->hist);
        h->hist_cap = h->opt.max_iters + 2;
        CK(dalloc((void **)&h->hist, (size_t)h->hist_cap * sizeof(double)));
    }
    int prec = solve_precision(h);
    int rc = ensure_vectors(h, prec);
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
    h->graphs.clear();
    // V-cycle parameters are read when its launches are enqueued (the graphs were just dropped)
    const int pre0_was = h->mg.pre0;
    mg_params(h);
    if (pre0_was && !h->mg.pre0 && h->mg.nlev > 0 && h->mg.lev[0].x1) { // the finest x1 must read as zero from now on
        cudaDeviceSynchronize();
        cudaMemset(h->mg.lev[0].x1, 0, (size_t)h->mg.lev[0].d.npad * sizeof(float));
        cudaDeviceSynchronize(); // complete before work on any stream, non-blocking ones included
    }
    return rc;
}

// ---------------------------------------------------------------------------
// One BiCGStab iteration, enqueued on stream s (captured into the graphs).
// ---------------------------------------------------------------------------
template <typename VT>
static void enqueue_precond(hicarw_handle *h, const VT *in, VT *out, int sweeps, SolveState *gate, int set_halt,
                            cudaStream_t s)
{
    OpCtx c = opctx(h);
    VT *Dinv = V<VT>(h, V_DINV), *pres = V<VT>(h, V_PRES);
    launch_precond_scale<VT>(h->d, in, out, Dinv, gate, set_halt, s);
    for (int sw = 2; sw <= sweeps; sw++) {
        launch_spmv<VT>(c, out, pres, gate, s);
        launch_rich<VT>(h->d, in, out, pres, Dinv, gate, s);
    }
}

template <typename VT, typename XT>
static void enqueue_iteration(hicarw_handle *h, XT *x, int sweeps, cudaStream_t s)
{
    OpCtx c = opctx(h);
    RedBuf rb{h->partials, h->red_blocks};
    SolveState *st = h->st;
    VT *r = V<VT>(h, V_R), *rhat = V<VT>(h, V_RHAT), *p = V<VT>(h, V_P), *phat = V<VT>(h, V_PHAT), *v = V<VT>(h, V_V),
       *sv = V<VT>(h, V_S), *shat = V<VT>(h, V_SHAT), *t = V<VT>(h, V_T), *Dinv = V<VT>(h, V_DINV),
       *pres = V<VT>(h, V_PRES);
    if (h->use_mg) { // multigrid-preconditioned BiCGStab (same recurrences, M = V-cycle)
        launch_iteration_begin(st, s);
        mg_apply<VT>(h->mg, p, phat, st, s);
        launch_spmv_sigma<VT>(c, phat, v, rhat, st, rb, s);
        launch_s_update<VT>(h->d, r, v, sv, st, s);
        mg_apply<VT>(h->mg, sv, shat, st, s);
        launch_spmv_dot5<VT>(c, shat, t, sv, rhat, st, h->hist, rb, s);
        launch_update_xrp<VT, XT>(h->d, x, phat, shat, r, sv, t, p, v, st, s);
        return;
    }
    enqueue_precond<VT>(h, p, phat, sweeps, st, 1, s);                 // :649
    launch_spmv_sigma<VT>(c, phat, v, rhat, st, rb, s);                // :657-688
    launch_s_precond<VT>(h->d, r, v, sv, shat, Dinv, st, s);           // :690 + sweep 1 of :695
    for (int sw = 2; sw <= sweeps; sw++) {
        launch_spmv<VT>(c, shat, pres, st, s);
        launch_rich<VT>(h->d, sv, shat, pres, Dinv, st, s);
    }
    launch_spmv_dot5<VT>(c, shat, t, sv, rhat, st, h->hist, rb, s);    // :703-750
    launch_update_xrp<VT, XT>(h->d, x, phat, shat, r, sv, t, p, v, st, s); // :755-783
}

// One iteration of the reference schedule in the vector precision prec.
static void enqueue_iteration_prec(hicarw_handle *h, int prec, int sweeps, cudaStream_t s)
{
    if (prec == HICARW_KRYLOV_F64) enqueue_iteration<double, double>(h, V<double>(h, V_X), sweeps, s);
    else enqueue_iteration<float, double>(h, V<double>(h, V_X), sweeps, s);
}

// The set-up kernel (r = b - A x, r^ = p = r and the first dots) in the vector
// precision prec; restart != 0 keeps the iteration count and the target.
static void enqueue_setup_prec(hicarw_handle *h, int prec, const OpCtx &c, const RedBuf &rb, cudaStream_t s,
                               int restart)
{
    if (prec == HICARW_KRYLOV_F64)
        launch_setup<double, double>(c, V<double>(h, V_X), V<double>(h, V_RHS), V<double>(h, V_R),
                                     V<double>(h, V_RHAT), V<double>(h, V_P), h->st, h->hist, rb, restart, s);
    else
        launch_setup<float, double>(c, V<double>(h, V_X), V<float>(h, V_RHS), V<float>(h, V_R), V<float>(h, V_RHAT),
                                    V<float>(h, V_P), h->st, h->hist, rb, restart, s);
}

// FP64 true residual of the current solution in the vector precision prec:
// mode 0 the norm only (-> true_res), 1 residual replacement (r = b - A x and
// rho = <r^, r>; nothing once the solve has stopped).
static void enqueue_true_residual_prec(hicarw_handle *h, int prec, int mode, cudaStream_t s)
{
    OpCtx c = opctx(h);
    RedBuf rb{h->partials, h->red_blocks};
    if (prec == HICARW_KRYLOV_F64)
        launch_true_residual<double, double>(c, V<double>(h, V_X), V<double>(h, V_RHS), mode ? V<double>(h, V_R) : nullptr,
                                             mode ? V<double>(h, V_RHAT) : nullptr, h->st, mode, rb, s);
    else
        launch_true_residual<float, double>(c, V<double>(h, V_X), V<float>(h, V_RHS), mode ? V<float>(h, V_R) : nullptr,
                                            mode ? V<float>(h, V_RHAT) : nullptr, h->st, mode, rb, s);
}

static int get_graph(hicarw_handle *h, int prec, int sweeps, int chunk, GraphRec **out)
{
    GraphKey key{prec, sweeps, chunk, h->opt.solver, h->opt.replace_every, h->use_mg};
    auto it = h->graphs.find(key);
    if (it != h->graphs.end()) { *out = &it->second; return 0; }
    cudaGraph_t graph;
    g_capturing = 1;
    g_capture_nodes = 0;
    CK(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
    for (int q = 0; q < chunk; q++) enqueue_iteration_prec(h, prec, sweeps, h->cap);
    cudaError_t e = cudaStreamEndCapture(h->cap, &graph);
    g_capturing = 0;
    if (e != cudaSuccess) { set_err(h, "cudaStreamEndCapture", e); return HICARW_ERR_CUDA; }
    GraphRec rec;
    rec.nodes = g_capture_nodes;
    e = cudaGraphInstantiate(&rec.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { set_err(h, "cudaGraphInstantiate", e); return HICARW_ERR_CUDA; }
    auto res = h->graphs.emplace(key, rec);
    *out = &res.first->second;
    return 0;
}

// Run the BiCGStab loop until the device says stop.  Returns the reference
// status (0/1/2) in h->hst after the call.
static int run_loop(hicarw_handle *h, int prec, int sweeps, cudaStream_t s)
{
    GraphRec *g = nullptr;
    int chunk = h->opt.check_every;
    int rc = get_graph(h, prec, sweeps, chunk, &g);
    if (rc) return rc;
    const int max_chunks = (h->opt.max_iters + chunk - 1) / chunk + 2;
    // FP32 Krylov vectors: the recurrence residual is replaced by the FP64 true
    // residual of the FP64 solution every replace_every iterations (rounded to graphs)
    const int rep = prec != HICARW_KRYLOV_F64 && h->opt.replace_every > 0 ? std::max(1, h->opt.replace_every / chunk) : 0;
    h->hflag[0] = h->hflag[1] = 0;
    for (int n = 0; n < max_chunks; n++) {
        CK(cudaGraphLaunch(g->exec, s));
        g_launches += g->nodes;
        if (rep && (n + 1) % rep == 0) enqueue_true_residual_prec(h, prec, 1, s);
        CK(cudaMemcpyAsync(&h->hflag[n & 1], &h->st->stop, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaEventRecord(h->ev[n & 1], s));
        if (n >= 1) {
            CK(cudaEventSynchronize(h->ev[(n - 1) & 1]));
            if (h->hflag[(n - 1) & 1]) break;
        }
    }
    return 0;
}

// The device state after a solve, copied to the pinned mirror.
static int fetch_state(hicarw_handle *h, cudaStream_t s)
{
    CK(cudaMemcpyAsync(h->hst, h->st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h->hst->err) {
        h->err = "a bounded device-side wait timed out (multigrid smoother copies)";
        return HICARW_ERR_TIMEOUT;
    }
    return 0;
}

// bicgstab_solve (:555-791) on the current x / rhs.  Fills st (pinned mirror).
static int fgmres_solve(hicarw_handle *h, int sweeps, cudaStream_t s);

// Preconditioner of a solve: the V-cycle (HICARW_PRECOND_MG, and the first
// stage of HICARW_PRECOND_MG_LEARNED), the U-Net alone (HICARW_PRECOND_LEARNED),
// or the V-cycle followed by the U-Net's correction of the residual it leaves
// (HICARW_PRECOND_MG_LEARNED); the forms with the U-Net run inside FGMRES only,
// and all but Jacobi need the probed operator.
static void select_precond(hicarw_handle *h, int allow)
{
    const int p = h->opt.precond;
    const bool fg = h->opt.solver == HICARW_SOLVER_FGMRES, ok = allow && h->operator_probed;
    h->use_mglearned = ok && fg && p == HICARW_PRECOND_MG_LEARNED && h->unet != nullptr;
    h->use_mg = ok && (p == HICARW_PRECOND_MG || h->use_mglearned);
    h->use_learned = ok && fg && p == HICARW_PRECOND_LEARNED && h->unet != nullptr;
}
static int precond_kind(const hicarw_handle *h)
{
    return h->use_mglearned ? HICARW_PRECOND_MG_LEARNED
                            : h->use_learned ? HICARW_PRECOND_LEARNED
                                             : h->use_mg ? HICARW_PRECOND_MG : HICARW_PRECOND_JACOBI;
}

// prec >= 0: the Krylov vector precision of this solve instead of the options'
// (the vectors, the right-hand side and the diagonal must already be in it).
static int bicgstab_solve(hicarw_handle *h, int sweeps, cudaStream_t s, int allow_mg = 1, int prec_in = -1)
{
    int rc;
    select_precond(h, allow_mg);
    if (h->use_mg && (h->mg_dirty || !h->mg.ready)) {
        mg_params(h);
        if (mg_build_tuned(h, s) != 0) { h->err = "multigrid build failed"; return HICARW_ERR_CUDA; }
        h->mg_dirty = 0;
    }
    if (h->opt.solver == HICARW_SOLVER_FGMRES) return fgmres_solve(h, sweeps, s);
    const int solver = h->opt.solver;
    const int prec = prec_in >= 0 ? prec_in : solve_precision(h);
    rc = ensure_vectors(h, prec);
    if (rc) return rc;
    OpCtx c = opctx(h);
    RedBuf rb{h->partials, h->red_blocks};
    launch_state_reset(h->st, h->opt.tol_rel, h->opt.tol_abs, h->opt.max_iters,
                       h->use_mg ? h->opt.stall_iters : 0, s);
    CK(cudaEventRecord(h->t0, s));
    (void)solver;
    enqueue_setup_prec(h, prec, c, rb, s, 0);
    rc = run_loop(h, prec, sweeps, s);
    if (rc) return rc;
    // true-residual stopping rule (iterative refinement of lambda): while the
    // FP64 residual of the FP64 solution is above the target, restart the
    // recurrences from it (r = r^ = p = b - A x) and continue
    if (h->opt.criterion == HICARW_CRIT_TRUE) {
        for (int rs = 0; rs < 20; rs++) {
            if ((rc = fetch_state(h, s)) != 0) return rc;
            if (h->hst->status != 0) break;
            enqueue_true_residual_prec(h, prec, 0, s);
            if ((rc = fetch_state(h, s)) != 0) return rc;
            if (h->hst->true_res <= h->hst->target || h->hst->it >= h->opt.max_iters) break;
            enqueue_setup_prec(h, prec, c, rb, s, 1);
            rc = run_loop(h, prec, sweeps, s);
            if (rc) return rc;
        }
    }
    CK(cudaEventRecord(h->t1, s));
    // final FP64 true residual of the solution (diagnostic; reference has none)
    enqueue_true_residual_prec(h, prec, 0, s);
    return fetch_state(h, s);
}

// ---- flexible GMRES ------------------------------------------------------------
namespace hw { // k_unet.cu
int unet_prepare_operator(hicarw_unet *n, const OpCtx &c, cudaStream_t s);
int unet_precond(hicarw_unet *n, const OpCtx &c, const double *in, double *out, const SolveState *gate, cudaStream_t s);
bool unet_matches(const hicarw_unet *n, const Dims &d);
}  // namespace hw

// z = M(r) + theta U(r'), r' = r - A M(r): the V-cycle, then the U-Net's
// estimate of the error left in the residual r' that the V-cycle leaves, taken
// with the minimal-residual step theta = <r', A u> / <A u, A u> (u = U(r')), so
// that ||r - A z|| = min over theta of ||r' - theta A u|| <= ||r'||: the composite
// never leaves a larger residual than the V-cycle alone, whatever the network
// returns.  Scratch: V_T (A M(r), then u), V_PRES (r'), V_V (A u); all three are
// free during FGMRES.
__global__ void mgl_residual_kernel(long long n, const double *__restrict__ r, double *__restrict__ az,
                                    double *__restrict__ res, const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        res[q] = r[q] - az[q];
        az[q] = 0.0; // the U-Net writes the interior of its output only
    }
}

// theta = <r', A u> / <A u, A u> (0 when A u = 0), left in st->mr_theta by the last CTA
__global__ void __launch_bounds__(256) mgl_step_kernel(long long n, const double *__restrict__ res,
                                                       const double *__restrict__ au, SolveState *st,
                                                       double *partials, const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    double acc[2] = {0.0, 0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const double a = au[q];
        acc[0] += res[q] * a;
        acc[1] += a * a;
    }
    double tot[2];
    if (!grid_reduce<2>(acc, partials, &st->ticket[5], tot)) return;
    if (threadIdx.x == 0) st->mr_theta = tot[1] > 0.0 ? tot[0] / tot[1] : 0.0;
}

__global__ void mgl_add_kernel(long long n, const double *__restrict__ u, double *__restrict__ z, const SolveState *st,
                               const SolveState *gate)
{
    if (gate && *(volatile const int *)&gate->stop && !gate->profile) return;
    const double theta = st->mr_theta;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        z[q] += theta * u[q];
}

static void mg_learned_apply(hicarw_handle *h, const double *in, double *out, const SolveState *gate, cudaStream_t s)
{
    const OpCtx c = opctx(h);
    const long long n = h->d.npad;
    const int g = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    const int gr = std::min(g, h->red_blocks);
    double *az = V<double>(h, V_T), *res = V<double>(h, V_PRES), *au = V<double>(h, V_V);
    mg_apply<double>(h->mg, in, out, gate, s);
    launch_spmv<double>(c, out, az, gate, s);
    {
        ProfScope ps_("mgl_residual", (double)n * 32.0, s);
        mgl_residual_kernel<<<g, 256, 0, s>>>(n, in, az, res, gate);
        count_launch(1);
    }
    unet_precond(h->unet, c, res, az, gate, s);
    launch_spmv<double>(c, az, au, gate, s);
    {
        ProfScope ps_("mgl_step", (double)n * 16.0, s);
        mgl_step_kernel<<<gr, 256, 0, s>>>(n, res, au, h->st, h->partials, gate);
        count_launch(1);
    }
    ProfScope ps_("mgl_add", (double)n * 24.0, s);
    mgl_add_kernel<<<g, 256, 0, s>>>(n, az, out, h->st, gate);
    count_launch(1);
}

static void fgmres_precond_cb(void *ctx, const double *in, double *out, cudaStream_t s)
{
    auto *pc = (decltype(hicarw_handle::fg_pc) *)ctx;
    hicarw_handle *h = pc->h;
    if (h->use_mglearned) mg_learned_apply(h, in, out, h->st, s);
    else if (h->use_learned) unet_precond(h->unet, opctx(h), in, out, h->st, s);
    else if (h->use_mg) mg_apply<double>(h->mg, in, out, h->st, s);
    else enqueue_precond<double>(h, in, out, pc->sweeps, h->st, 0, s);
}

// Buffers (sized for the restart length) and the launch context of FGMRES(m).
static int fgmres_prepare(hicarw_handle *h, int sweeps, FgmresCtx *f)
{
    int rc = ensure_vectors(h, HICARW_KRYLOV_F64);
    if (rc) return rc;
    const Dims &d = h->d;
    int m = h->opt.fgmres_restart;
    if (m < 1) m = 1;
    if (m > FG_MAXM) m = FG_MAXM;
    if (!h->gst) CK(dalloc((void **)&h->gst, sizeof(GmresState)));
    if (!h->fg_host) CK(cudaMallocHost((void **)&h->fg_host, sizeof(GmresState)));
    if (h->fg_m != m) {
        if (h->fgV) cudaFree(h->fgV);
        if (h->fgZ) cudaFree(h->fgZ);
        if (h->fgW) cudaFree(h->fgW);
        h->fgV = h->fgZ = h->fgW = nullptr;
        CK(dalloc((void **)&h->fgV, (size_t)(m + 1) * d.npad * sizeof(double)));
        CK(dalloc((void **)&h->fgZ, (size_t)m * d.npad * sizeof(double)));
        CK(dalloc((void **)&h->fgW, (size_t)d.npad * sizeof(double)));
        h->fg_m = m;
        for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
        h->graphs.clear();
    }
    h->fg_pc.h = h;
    h->fg_pc.sweeps = sweeps;
    f->op = opctx(h);
    f->m = m;
    f->x = V<double>(h, V_X);
    f->b = V<double>(h, V_RHS);
    f->V = h->fgV;
    f->Z = h->fgZ;
    f->W = h->fgW;
    f->partials = h->partials;
    f->red_blocks = h->red_blocks;
    f->dot_blocks = 296;
    f->g = h->gst;
    f->g_h1 = h->gst->h1;
    f->g_h2 = h->gst->h2;
    f->g_hnext = &h->gst->hnext;
    f->precond = fgmres_precond_cb;
    f->pctx = &h->fg_pc;
    return 0;
}

static void fgmres_enqueue_cycle(const FgmresCtx &f, cudaStream_t s)
{
    fgmres_enqueue_restart(f, s);
    for (int j = 0; j < f.m; j++) fgmres_enqueue_step(f, j, s);
    fgmres_enqueue_finish(f, s);
}

// buffers, launch context and (learned preconditioner) operator features of an FGMRES solve
static int fgmres_ready(hicarw_handle *h, int sweeps, cudaStream_t s, FgmresCtx *f)
{
    int rc = fgmres_prepare(h, sweeps, f);
    if (rc) return rc;
    if ((h->use_learned || h->use_mglearned) && h->unet_dirty) {
        if (unet_prepare_operator(h->unet, opctx(h), s) != 0) {
            h->err = "learned preconditioner grid mismatch";
            return HICARW_ERR_ARG;
        }
        h->unet_dirty = 0;
    }
    return 0;
}

// the FGMRES device state mapped onto the solve-state mirror (stats), with the
// FP64 true residual of the solution
static int fgmres_map_state(hicarw_handle *h, int stalled, cudaStream_t s)
{
    GmresState gh;
    CK(cudaMemcpyAsync(&gh, h->gst, sizeof(GmresState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    OpCtx c = opctx(h);
    RedBuf rb{h->partials, h->red_blocks};
    launch_true_residual<double, double>(c, V<double>(h, V_X), V<double>(h, V_RHS), nullptr, nullptr, h->st, 0, rb, s);
    int rc;
    if ((rc = fetch_state(h, s)) != 0) return rc;
    h->hst->status = stalled ? 4 : gh.status;
    h->hst->it = gh.it_total;
    h->hst->res0 = gh.res0;
    h->hst->rnorm = gh.res;
    h->hst->bnorm2 = gh.bnorm * gh.bnorm;
    h->hst->target = gh.target;
    return 0;
}

static int fgmres_solve(hicarw_handle *h, int sweeps, cudaStream_t s)
{
    FgmresCtx f;
    int rc = fgmres_ready(h, sweeps, s, &f);
    if (rc) return rc;
    const int m = f.m;
    fgmres_reset(h->gst, m, h->opt.tol_rel, h->opt.tol_abs, h->opt.max_iters, h->hist, h->st, s);
    CK(cudaEventRecord(h->t0, s));
    // one restart cycle = one graph
    const int pkind = precond_kind(h);
    GraphKey key{HICARW_KRYLOV_F64, sweeps, m, HICARW_SOLVER_FGMRES, 0, pkind};
    auto it = h->graphs.find(key);
    if (it == h->graphs.end()) {
        cudaGraph_t graph;
        g_capturing = 1;
        g_capture_nodes = 0;
        CK(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
        fgmres_enqueue_cycle(f, h->cap);
        cudaError_t e = cudaStreamEndCapture(h->cap, &graph);
        g_capturing = 0;
        if (e != cudaSuccess) { set_err(h, "capture fgmres", e); return HICARW_ERR_CUDA; }
        GraphRec rec;
        rec.nodes = g_capture_nodes;
        e = cudaGraphInstantiate(&rec.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { set_err(h, "instantiate fgmres", e); return HICARW_ERR_CUDA; }
        it = h->graphs.emplace(key, rec).first;
    }
    const int max_cycles = h->opt.max_iters / m + 2;
    GmresState *hg = h->fg_host;
    double best = 0.0;
    int best_it = 0, stalled = 0;
    for (int c = 0; c < max_cycles; c++) {
        CK(cudaGraphLaunch(it->second.exec, s));
        g_launches += it->second.nodes;
        CK(cudaMemcpyAsync(hg, h->gst, offsetof(GmresState, hist), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (hg->status == 0 || hg->it_total >= hg->max_iters) break;
        // stall detector (as for BiCGStab): no 1% decrease of the residual within stall_iters steps
        if (c == 0 || hg->res < 0.99 * best) {
            best = hg->res;
            best_it = hg->it_total;
        } else if (h->opt.stall_iters > 0 && hg->it_total - best_it >= h->opt.stall_iters) {
            stalled = 1;
            break;
        }
        // not converged within the cycle: the next launch restarts from the current x
    }
    CK(cudaEventRecord(h->t1, s));
    return fgmres_map_state(h, stalled, s);
}

static void fill_stats(hicarw_handle *h, hicarw_stats *o, int sweeps, int retries)
{
    if (!o) return;
    const SolveState *st = h->hst;
    o->status = st->status;
    o->iterations = st->it;
    o->sweeps = sweeps;
    o->retries = retries;
    o->res0 = st->res0;
    o->res_final = st->rnorm;
    o->b_norm = sqrt(st->bnorm2);
    o->target = st->target;
    o->true_res = st->true_res;
    o->replacements = st->replacements;
    o->precond = precond_kind(h);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, h->t0, h->t1);
    o->solve_ms = ms;
    o->launches = (int)(g_launches.load() - h->launches_at_call);
}

// lambda used by the wind correction: x (REFERENCE) or the FP64 accumulator.
static int enqueue_winds(hicarw_handle *h, const float *rho, int adv_den, float *u, float *v, float *w, cudaStream_t s)
{
    Metrics m = metrics_of(h);
    launch_winds<double>(h->d, m, V<double>(h, V_X), h->alpha, rho, u, v, w, adv_den, s);
    return 0;
}

static int zero_solution(hicarw_handle *h, cudaStream_t s)
{
    CK(cudaMemsetAsync(h->vec[V_X], 0, (size_t)h->d.npad * 8, s));
    return 0;
}

extern "C" int hicarw_reset_solution(hicarw_handle *h, void *stream)
{
    api_entry();
    if (!h) return HICARW_ERR_ARG;
    return zero_solution(h, (cudaStream_t)stream);
}

// extract_diagonal + compute_rhs_3d (:430, :433) for the current state.
static void prepare_system(hicarw_handle *h, cudaStream_t s)
{
    const Dims &d = h->d;
    if (h->vprec == HICARW_KRYLOV_F64) {
        launch_diag<double>(d, h->coef, h->dz_if, V<double>(h, V_DINV), h->operator_probed, s);
        launch_rhs<double>(d, h->div, V<double>(h, V_RHS), s);
    } else {
        launch_diag<float>(d, h->coef, h->dz_if, V<float>(h, V_DINV), h->operator_probed, s);
        launch_rhs<float>(d, h->div, V<float>(h, V_RHS), s);
    }
}

extern "C" int hicarw_calc_iter_winds(hicarw_handle *h, const float *alpha, const float *div, const float *density,
                                      int adv_den, float *u, float *v, float *w, int mem_kind, void *stream,
                                      hicarw_stats *stats)
{
    api_entry();
    if (!h || !alpha || !div || !u || !v || !w || (adv_den && !density)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    h->launches_at_call = g_launches.load();
    int rc;
    const int prec = solve_precision(h);
    if ((rc = ensure_vectors(h, prec)) != 0) return rc;
    // module copies of alpha and div (:308-317)
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpyAsync(h->alpha, alpha, n_cell(d) * 4, kind, s));
    CK(cudaMemcpyAsync(h->div, div, n_cell(d) * 4, kind, s));
    const float *rho = nullptr, *du = nullptr, *dv = nullptr, *dw = nullptr;
    if (adv_den && (rc = stage_in(h, density, &h->srho, n_cell(d), mem_kind, s, &rho)) != 0) return rc;
    if ((rc = stage_in(h, u, &h->su, n_u(d), mem_kind, s, &du)) != 0) return rc;
    if ((rc = stage_in(h, v, &h->sv, n_v(d), mem_kind, s, &dv)) != 0) return rc;
    if ((rc = stage_in(h, w, &h->sw, n_cell(d), mem_kind, s, &dw)) != 0) return rc;
    // NaN scan of div and alpha min/max (:319-329, :411-421): one pass, read back once
    CK(cudaMemsetAsync(h->scan, 0, 3 * sizeof(unsigned int), s));
    CK(cudaMemsetAsync(h->scan + 1, 0xff, sizeof(unsigned int), s));
    launch_scan_inputs((long long)n_cell(d), h->div, h->alpha, h->scan, s);
    CK(cudaMemcpyAsync(h->hscan, h->scan, 3 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    if (!h->structure_uploaded) { // first call: analytic coefficients (:351-407)
        launch_coefs(d, metrics_of(h), h->alpha, h->coef, 0, s);
        launch_bccol(d, metrics_of(h), h->alpha, h->bc, s);
        if ((rc = zero_solution(h, s)) != 0) return rc;
        h->structure_uploaded = 1;
        h->mg_dirty = h->unet_dirty = 1;
        CK(cudaStreamSynchronize(s));
    } else {
        CK(cudaStreamSynchronize(s));
        unsigned int bmn = h->hscan[1], bmx = h->hscan[2];
        if (bmx > bmn && !h->operator_probed) { // varying alpha -> update_coefs_gpu (:423-426)
            launch_coefs(d, metrics_of(h), h->alpha, h->coef, 1, s);
            launch_bccol(d, metrics_of(h), h->alpha, h->bc, s);
            h->mg_dirty = h->unet_dirty = 1;
        }
    }
    if (h->hscan[0] > 0 && h->opt.verbose)
        fprintf(stderr, "HICAR wind solver: NaN in input divergence (count=%u)\n", h->hscan[0]);
    prepare_system(h, s);
    int sweeps = h->precond_n_sweeps;
    if ((rc = bicgstab_solve(h, sweeps, s)) != 0) return rc;
    int fell_back = 0;
    if ((h->use_mg || h->use_learned) && h->hst->status != 0) { // preconditioned solve stalled or failed: the reference solve decides
        if (h->opt.verbose)
            fprintf(stderr, " HICAR multigrid BiCGStab status=%d after %d iterations: falling back to Jacobi\n",
                    h->hst->status, h->hst->it);
        // the reference's method in the reference's precision: with FP32 vectors
        // the Jacobi-preconditioned recurrences can drift to NaN on hard systems
        if ((rc = ensure_vectors(h, HICARW_KRYLOV_F64)) != 0) return rc;
        prepare_system(h, s);
        if ((rc = zero_solution(h, s)) != 0) return rc;
        if ((rc = bicgstab_solve(h, sweeps, s, 0, HICARW_KRYLOV_F64)) != 0) return rc;
        fell_back = 1;
    }
    int retries = 0;
    double res0 = h->hst->res0, resf = h->hst->rnorm;
    int status = h->hst->status, iters = h->hst->it;
    if (h->opt.verbose)
        fprintf(stderr, " HICAR BiCGStab status=%d iterations=%d precond_n_sweeps=%d res0=%g res_final=%g\n", status,
                iters, sweeps, res0, resf);
    // adaptive sweep retry (:479-503)
    if (status != 0 && iters > 0 && resf > 0.01 * res0) {
        while (status != 0 && resf > 0.01 * res0 && h->precond_n_sweeps < MAX_PREC_SWEEPS) {
            h->precond_n_sweeps++;
            sweeps = h->precond_n_sweeps;
            if ((rc = zero_solution(h, s)) != 0) return rc;
            if ((rc = fell_back ? bicgstab_solve(h, sweeps, s, 0, HICARW_KRYLOV_F64) : bicgstab_solve(h, sweeps, s)) != 0)
                return rc;
            retries++;
            res0 = h->hst->res0; resf = h->hst->rnorm; status = h->hst->status; iters = h->hst->it;
            if (h->opt.verbose)
                fprintf(stderr, "  Retry status=%d iterations=%d sweeps=%d\n", status, iters, sweeps);
        }
        h->precond_n_sweeps = BASE_PREC_SWEEPS;
        if (status != 0 && resf > res0) { // the reference stops the model here (:506-528)
            fill_stats(h, stats, sweeps, retries);
            h->err = "BiCGStab diverged after every preconditioner retry";
            return HICARW_ERR_DIVERGED;
        }
    }
    enqueue_winds(h, rho, adv_den, (float *)du, (float *)dv, (float *)dw, s); // :531
    if (mem_kind == HICARW_MEM_HOST) {
        CK(cudaMemcpyAsync(u, du, n_u(d) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(v, dv, n_v(d) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(w, dw, n_cell(d) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    fill_stats(h, stats, sweeps, retries);
    if (fell_back && status == 0) {
        if (stats) stats->status = HICARW_FELL_BACK;
        return HICARW_FELL_BACK;
    }
    return status;
}

extern "C" int hicarw_calc_divergence(hicarw_handle *h, const float *u, const float *v, const float *w,
                                      const float *density, float *div, int adv_den, int horz_only, int use_dqdt,
                                      int mem_kind, void *stream)
{
    api_entry();
    if (!h || !u || !v || !w || !div || (adv_den && !density)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    const float *du, *dv, *dw, *rho = nullptr;
    int rc;
    if ((rc = stage_in(h, u, &h->su, n_u(d), mem_kind, s, &du)) != 0) return rc;
    if ((rc = stage_in(h, v, &h->sv, n_v(d), mem_kind, s, &dv)) != 0) return rc;
    if ((rc = stage_in(h, w, &h->sw, n_cell(d), mem_kind, s, &dw)) != 0) return rc;
    if (adv_den && (rc = stage_in(h, density, &h->srho, n_cell(d), mem_kind, s, &rho)) != 0) return rc;
    float *ddiv = div;
    if (mem_kind == HICARW_MEM_HOST) {
        if (!h->sdiv) CK(cudaMalloc((void **)&h->sdiv, n_cell(d) * 4));
        ddiv = h->sdiv;
    }
    launch_divergence(d, metrics_of(h), du, dv, dw, rho, ddiv, adv_den, horz_only, use_dqdt, s);
    if (mem_kind == HICARW_MEM_HOST) {
        CK(cudaMemcpyAsync(div, ddiv, n_cell(d) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    return HICARW_OK;
}

// ---- probing -------------------------------------------------------------
extern "C" int hicarw_probe_lambda_pattern(hicarw_handle *h, int ca, int cb, int cc, void *stream)
{
    api_entry();
    if (!h || ca < 0 || ca > 2 || cb < 0 || cb > 2 || cc < 0 || cc > 2) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    launch_probe_pattern<double>(h->d, V<double>(h, V_X), ca, cb, cc, s);
    return HICARW_OK;
}

extern "C" int hicarw_probe_zero_corrections(hicarw_handle *h, float *u, float *v, float *w, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !u || !v || !w) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    if (mem_kind == HICARW_MEM_HOST) {
        memset(u, 0, n_u(d) * 4); memset(v, 0, n_v(d) * 4); memset(w, 0, n_cell(d) * 4);
        return HICARW_OK;
    }
    CK(cudaMemsetAsync(u, 0, n_u(d) * 4, s));
    CK(cudaMemsetAsync(v, 0, n_v(d) * 4, s));
    CK(cudaMemsetAsync(w, 0, n_cell(d) * 4, s));
    return HICARW_OK;
}

// calc_updated_winds from the current x_sol (probe_apply_corrections, :1158-1163).
extern "C" int hicarw_probe_apply_corrections(hicarw_handle *h, const float *alpha, const float *density, int adv_den,
                                              float *u, float *v, float *w, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !alpha || !u || !v || !w || (adv_den && !density)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpyAsync(h->alpha, alpha, n_cell(d) * 4, kind, s));
    const float *rho = nullptr, *du, *dv, *dw;
    int rc;
    if (adv_den && (rc = stage_in(h, density, &h->srho, n_cell(d), mem_kind, s, &rho)) != 0) return rc;
    if ((rc = stage_in(h, u, &h->su, n_u(d), mem_kind, s, &du)) != 0) return rc;
    if ((rc = stage_in(h, v, &h->sv, n_v(d), mem_kind, s, &dv)) != 0) return rc;
    if ((rc = stage_in(h, w, &h->sw, n_cell(d), mem_kind, s, &dw)) != 0) return rc;
    Metrics m = metrics_of(h);
    launch_winds<double>(d, m, V<double>(h, V_X), h->alpha, rho, (float *)du, (float *)dv, (float *)dw, adv_den, s);
    if (mem_kind == HICARW_MEM_HOST) {
        CK(cudaMemcpyAsync(u, du, n_u(d) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(v, dv, n_v(d) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(w, dw, n_cell(d) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    return HICARW_OK;
}

extern "C" int hicarw_probe_record(hicarw_handle *h, const float *Tfield, int ca, int cb, int cc, float *max_leak,
                                   int mem_kind, void *stream)
{
    api_entry();
    if (!h || !Tfield || !max_leak) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const float *T;
    int rc;
    if ((rc = stage_in(h, Tfield, &h->sT, n_cell(h->d), mem_kind, s, &T)) != 0) return rc;
    unsigned int bits;
    memcpy(&bits, max_leak, 4);
    h->hscan[3] = bits;
    CK(cudaMemcpyAsync(h->scan + 3, &h->hscan[3], 4, cudaMemcpyHostToDevice, s));
    launch_probe_record(h->d, T, h->coef, ca, cb, cc, h->scan + 3, s);
    CK(cudaMemcpyAsync(&h->hscan[3], h->scan + 3, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    memcpy(max_leak, &h->hscan[3], 4);
    return HICARW_OK;
}

extern "C" int hicarw_probe_finalize(hicarw_handle *h, float max_leak, void *stream)
{
    api_entry();
    if (!h) return HICARW_ERR_ARG;
    h->operator_probed = 1;
    h->structure_uploaded = 1;
    h->mg_dirty = h->unet_dirty = 1;
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
    h->graphs.clear();
    if (h->opt.verbose)
        fprintf(stderr, "Projection operator calibrated by probing (A = 2*D o G); off-stencil leakage max |T| = %g\n",
                (double)max_leak);
    return zero_solution(h, (cudaStream_t)stream); // :1243
}

extern "C" int hicarw_calibrate_projection_operator(hicarw_handle *h, const float *alpha, const float *density,
                                                    int adv_den, float *u, float *v, float *w, float *max_leak,
                                                    int mem_kind, void *stream)
{
    api_entry();
    if (!h || !alpha || !u || !v || !w || (adv_den && !density)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    int rc;
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpyAsync(h->alpha, alpha, n_cell(d) * 4, kind, s));
    const float *rho = nullptr;
    if (adv_den && (rc = stage_in(h, density, &h->srho, n_cell(d), mem_kind, s, &rho)) != 0) return rc;
    // scratch winds (the reference saves u/v/w dqdt, probes in them and restores them;
    // probing in separate buffers leaves the caller's arrays untouched, same result)
    if (!h->sprobe_u) {
        CK(cudaMalloc((void **)&h->sprobe_u, n_u(d) * 4));
        CK(cudaMalloc((void **)&h->sprobe_v, n_v(d) * 4));
        CK(cudaMalloc((void **)&h->sprobe_w, n_cell(d) * 4));
    }
    if (!h->sT) CK(cudaMalloc((void **)&h->sT, n_cell(d) * 4));
    if (!h->structure_uploaded) { // the analytic coefficients fill the rows a probe never reaches
        launch_coefs(d, metrics_of(h), h->alpha, h->coef, 0, s);
        launch_bccol(d, metrics_of(h), h->alpha, h->bc, s);
        h->structure_uploaded = 1;
    }
    CK(cudaMemsetAsync(h->scan + 3, 0, 4, s));
    Metrics m = metrics_of(h);
    for (int cc = 0; cc < 3; cc++)
        for (int cb = 0; cb < 3; cb++)
            for (int ca = 0; ca < 3; ca++) {
                launch_probe_pattern<double>(d, V<double>(h, V_X), ca, cb, cc, s);
                CK(cudaMemsetAsync(h->sprobe_u, 0, n_u(d) * 4, s));
                CK(cudaMemsetAsync(h->sprobe_v, 0, n_v(d) * 4, s));
                CK(cudaMemsetAsync(h->sprobe_w, 0, n_cell(d) * 4, s));
                launch_winds<double>(d, m, V<double>(h, V_X), h->alpha, rho, h->sprobe_u, h->sprobe_v, h->sprobe_w, adv_den, s);
                launch_divergence(d, m, h->sprobe_u, h->sprobe_v, h->sprobe_w, rho, h->sT, adv_den, 0, 1, s);
                launch_probe_record(d, h->sT, h->coef, ca, cb, cc, h->scan + 3, s);
            }
    CK(cudaMemcpyAsync(&h->hscan[3], h->scan + 3, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    float leak;
    memcpy(&leak, &h->hscan[3], 4);
    if (max_leak) *max_leak = leak;
    (void)u; (void)v; (void)w;
    return hicarw_probe_finalize(h, leak, stream);
}

// ---- extensions ----------------------------------------------------------
extern "C" int hicarw_get_lambda(hicarw_handle *h, double *lambda, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !lambda) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    size_t n = (size_t)d.mx * d.mz * d.my;
    double *gath = nullptr;
    CK(cudaMalloc((void **)&gath, n * 8));
    const double *src64 = V<double>(h, V_X);
    // gather the padded rows into the (nx+2, nz+2, ny+2) Fortran layout
    cudaError_t e = cudaMemcpy2DAsync(gath, sizeof(double) * d.mx, src64 + XO, sizeof(double) * d.P,
                                      sizeof(double) * d.mx, (size_t)d.mz * d.my, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(lambda, gath, n * 8,
                            mem_kind == HICARW_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(gath);
    if (e != cudaSuccess || e2 != cudaSuccess) { set_err(h, "get_lambda", e != cudaSuccess ? e : e2); return HICARW_ERR_CUDA; }
    return HICARW_OK;
}

extern "C" int hicarw_get_coefs(hicarw_handle *h, float *coefs, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !coefs) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    for (int c = 0; c < NCOEF; c++) {
        // interior rows (1..nx, 1..nz, 1..ny) -> (nx, nz, ny)
        for (int j = 1; j <= d.ny; j++)
            CK(cudaMemcpy2DAsync(coefs + (size_t)c * n_cell(d) + (size_t)(j - 1) * d.nx * d.nz, sizeof(float) * d.nx,
                                 h->coef + (size_t)c * d.npad + kidx(d, 1, 1, j), sizeof(float) * d.P,
                                 sizeof(float) * d.nx, d.nz, kind, s));
    }
    CK(cudaStreamSynchronize(s));
    return HICARW_OK;
}

extern "C" int hicarw_set_coefs(hicarw_handle *h, const float *coefs, int probed, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !coefs) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int c = 0; c < NCOEF; c++)
        for (int j = 1; j <= d.ny; j++)
            CK(cudaMemcpy2DAsync(h->coef + (size_t)c * d.npad + kidx(d, 1, 1, j), sizeof(float) * d.P,
                                 coefs + (size_t)c * n_cell(d) + (size_t)(j - 1) * d.nx * d.nz, sizeof(float) * d.nx,
                                 sizeof(float) * d.nx, d.nz, kind, s));
    h->operator_probed = probed ? 1 : 0;
    h->structure_uploaded = 1;
    h->mg_dirty = h->unet_dirty = 1;
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
    h->graphs.clear();
    CK(cudaStreamSynchronize(s));
    return HICARW_OK;
}

// Copy a (nx+2, nz+2, ny+2) FP64 array into / out of a padded device vector.
static int put_padded(hicarw_handle *h, const double *src, double *dst, int mem_kind, cudaStream_t s)
{
    const Dims &d = h->d;
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpy2DAsync(dst + XO, sizeof(double) * d.P, src, sizeof(double) * d.mx, sizeof(double) * d.mx,
                         (size_t)d.mz * d.my, kind, s));
    return 0;
}
static int get_padded(hicarw_handle *h, const double *src, double *dst, int mem_kind, cudaStream_t s)
{
    const Dims &d = h->d;
    cudaMemcpyKind kind = mem_kind == HICARW_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpy2DAsync(dst, sizeof(double) * d.mx, src + XO, sizeof(double) * d.P, sizeof(double) * d.mx,
                         (size_t)d.mz * d.my, kind, s));
    return 0;
}

extern "C" int hicarw_apply_operator(hicarw_handle *h, const double *x, double *y, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !x || !y) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    double *bx, *by;
    CK(dalloc((void **)&bx, (size_t)d.npad * 8));
    CK(dalloc((void **)&by, (size_t)d.npad * 8));
    int rc = put_padded(h, x, bx, mem_kind, s);
    if (!rc) {
        launch_spmv<double>(opctx(h), bx, by, nullptr, s);
        rc = get_padded(h, by, y, mem_kind, s);
    }
    cudaStreamSynchronize(s);
    cudaFree(bx);
    cudaFree(by);
    return rc;
}

extern "C" int hicarw_apply_precond(hicarw_handle *h, const double *x, double *y, int sweeps, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !x || !y) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    if (sweeps <= 0 && !h->operator_probed) return HICARW_ERR_STATE; // the V-cycle needs the probed operator
    const bool learned = sweeps < 0 && (h->opt.precond == HICARW_PRECOND_LEARNED ||
                                        h->opt.precond == HICARW_PRECOND_MG_LEARNED);
    if (learned && !h->unet) return HICARW_ERR_STATE;
    double *bx, *by, *bd, *bp;
    CK(dalloc((void **)&bx, (size_t)d.npad * 8));
    CK(dalloc((void **)&by, (size_t)d.npad * 8));
    CK(dalloc((void **)&bd, (size_t)d.npad * 8));
    CK(dalloc((void **)&bp, (size_t)d.npad * 8));
    int rc = put_padded(h, x, bx, mem_kind, s);
    if (!rc && learned) rc = ensure_vectors(h, HICARW_KRYLOV_F64); // scratch of the composite
    if (!rc && learned && h->unet_dirty) {
        if (unet_prepare_operator(h->unet, opctx(h), s) != 0) rc = HICARW_ERR_ARG;
        else h->unet_dirty = 0;
    }
    if (!rc && sweeps <= 0) {
        if ((h->mg_dirty || !h->mg.ready) && !(learned && h->opt.precond == HICARW_PRECOND_LEARNED)) {
            mg_params(h);
            if (mg_build_tuned(h, s) != 0) rc = HICARW_ERR_CUDA;
            else h->mg_dirty = 0;
        }
        if (!rc) {
            CK(cudaMemsetAsync(by, 0, (size_t)d.npad * 8, s));
            if (learned && h->opt.precond == HICARW_PRECOND_LEARNED) unet_precond(h->unet, opctx(h), bx, by, nullptr, s);
            else if (learned) mg_learned_apply(h, bx, by, nullptr, s);
            else mg_apply<double>(h->mg, bx, by, nullptr, s);
            rc = get_padded(h, by, y, mem_kind, s);
        }
        int herr = 0;
        if (!rc && cudaMemcpy(&herr, h->mg.err, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && herr) {
            h->err = "a bounded device-side wait timed out (multigrid smoother copies)";
            rc = HICARW_ERR_TIMEOUT;
        }
    } else if (!rc) {
        launch_diag<double>(d, h->coef, h->dz_if, bd, h->operator_probed, s);
        OpCtx c = opctx(h);
        launch_precond_scale<double>(d, bx, by, bd, nullptr, 0, s);
        for (int sw = 2; sw <= sweeps; sw++) {
            launch_spmv<double>(c, by, bp, nullptr, s);
            launch_rich<double>(d, bx, by, bp, bd, nullptr, s);
        }
        rc = get_padded(h, by, y, mem_kind, s);
    }
    cudaStreamSynchronize(s);
    cudaFree(bx); cudaFree(by); cudaFree(bd); cudaFree(bp);
    return rc;
}

extern "C" int hicarw_solve_rhs(hicarw_handle *h, const double *rhs, int mem_kind, void *stream, hicarw_stats *stats)
{
    api_entry();
    if (!h || !rhs) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const Dims &d = h->d;
    h->launches_at_call = g_launches.load();
    const int prec = solve_precision(h);
    int rc = ensure_vectors(h, prec);
    if (rc) return rc;
    double *b;
    CK(dalloc((void **)&b, (size_t)d.npad * 8));
    rc = put_padded(h, rhs, b, mem_kind, s);
    if (!rc) {
        if (h->vprec == HICARW_KRYLOV_F64) {
            CK(cudaMemcpyAsync(V<double>(h, V_RHS), b, (size_t)d.npad * 8, cudaMemcpyDeviceToDevice, s));
            launch_diag<double>(d, h->coef, h->dz_if, V<double>(h, V_DINV), h->operator_probed, s);
        } else {
            launch_convert<double, float>(d.npad, b, V<float>(h, V_RHS), s);
            launch_diag<float>(d, h->coef, h->dz_if, V<float>(h, V_DINV), h->operator_probed, s);
        }
        rc = bicgstab_solve(h, h->precond_n_sweeps, s);
    }
    cudaStreamSynchronize(s);
    cudaFree(b);
    if (rc) return rc;
    fill_stats(h, stats, h->precond_n_sweeps, 0);
    return h->hst->status;
}

extern "C" int hicarw_get_history(hicarw_handle *h, double *out, int cap)
{
    api_entry();
    if (!h) return HICARW_ERR_ARG;
    int n = h->hst->it + 1;
    if (out && cap > 0) {
        int m = n < cap ? n : cap;
        if (cudaMemcpy(out, h->hist, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return HICARW_ERR_CUDA;
    }
    return n;
}

extern "C" const char *hicarw_last_error(hicarw_handle *h) { return h ? h->err.c_str() : g_err_noh.c_str(); }

extern "C" long long hicarw_kernel_launches(void) { return g_launches.load(); }
extern "C" long long hicarw_mg_tma_launches(void) { return mg_tma_posts(); }

// ---- per-kernel profile of one solve iteration ------------------------------
__global__ void prof_state_kernel(SolveState *s, int on)
{
    s->profile = on;
    s->stop = 0;
    s->halt = 0;
    s->upd_r = s->upd_p = 1;
    s->it = 0;
}

extern "C" int hicarw_profile_iteration(hicarw_handle *h, int reps, char *names, double *ms, double *bytes,
                                        int *per_iter, int cap, void *stream)
{
    api_entry();
    if (!h || reps < 1 || cap < 1) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int solver = h->opt.solver;
    const int prec = solve_precision(h);
    int rc = ensure_vectors(h, prec);
    if (rc) return rc;
    select_precond(h, 1);
    if ((h->use_learned || h->use_mglearned) && h->unet_dirty) {
        if (unet_prepare_operator(h->unet, opctx(h), s) != 0) return HICARW_ERR_ARG;
        h->unet_dirty = 0;
    }
    if (h->use_mg && (h->mg_dirty || !h->mg.ready)) {
        if (mg_build_tuned(h, s) != 0) return HICARW_ERR_CUDA;
        h->mg_dirty = 0;
    }
    FgmresCtx fg;
    if (solver == HICARW_SOLVER_FGMRES) {
        if ((rc = fgmres_prepare(h, h->precond_n_sweeps, &fg)) != 0) return rc;
        fgmres_reset(h->gst, fg.m, h->opt.tol_rel, h->opt.tol_abs, h->opt.max_iters, h->hist, h->st, s);
        fgmres_set_profile(h->gst, 1, s);
    }
    if (solver == HICARW_SOLVER_REFERENCE) {
        // start from the set-up of a cold solve (x = 0, r = r^ = p = b), so that every
        // kernel of the profiled iterations does the work of a live iteration
        OpCtx c = opctx(h);
        RedBuf rb{h->partials, h->red_blocks};
        if ((rc = zero_solution(h, s)) != 0) return rc;
        launch_state_reset(h->st, h->opt.tol_rel, h->opt.tol_abs, h->opt.max_iters, 0, s);
        enqueue_setup_prec(h, prec, c, rb, s, 0);
    }
    prof_state_kernel<<<1, 1, 0, s>>>(h->st, 1);
    CK(cudaStreamSynchronize(s));
    for (auto &r : g_prof) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    g_prof.clear();
    g_prof_on = 1;
    for (int q = 0; q < reps; q++) {
        if (solver == HICARW_SOLVER_FGMRES) {
            fgmres_enqueue_cycle(fg, s);
        } else {
            enqueue_iteration_prec(h, prec, h->precond_n_sweeps, s);
        }
    }
    g_prof_on = 0;
    prof_state_kernel<<<1, 1, 0, s>>>(h->st, 0);
    if (solver == HICARW_SOLVER_FGMRES) fgmres_set_profile(h->gst, 0, s);
    CK(cudaStreamSynchronize(s));
    // aggregate by kernel name, in first-launch order
    std::vector<std::string> nm;
    std::vector<double> tot, by;
    std::vector<int> cnt;
    for (auto &r : g_prof) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, r.a, r.b);
        size_t q = 0;
        while (q < nm.size() && nm[q] != r.name) q++;
        if (q == nm.size()) { nm.push_back(r.name); tot.push_back(0.0); by.push_back(0.0); cnt.push_back(0); }
        tot[q] += t;
        by[q] += r.bytes;
        cnt[q] += 1;
    }
    for (auto &r : g_prof) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    g_prof.clear();
    int n = (int)nm.size() < cap ? (int)nm.size() : cap;
    for (int q = 0; q < n; q++) {
        if (names) { strncpy(names + 32 * q, nm[q].c_str(), 31); names[32 * q + 31] = 0; }
        if (ms) ms[q] = tot[q] / cnt[q];
        if (bytes) bytes[q] = by[q] / cnt[q];
        if (per_iter) per_iter[q] = cnt[q] / reps;
    }
    // the profiling pass overwrote the Krylov state: restart the next solve cold
    return zero_solution(h, s) ? HICARW_ERR_CUDA : n;
}

extern "C" int hicarw_set_learned_precond(hicarw_handle *h, hicarw_unet *n)
{
    api_entry();
    if (!h) return HICARW_ERR_ARG;
    if (n && !unet_matches(n, h->d)) {
        h->err = "learned preconditioner: network grid differs from the handle's";
        return HICARW_ERR_ARG;
    }
    if (h->unet != n) {
        cudaDeviceSynchronize();
        for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
        h->graphs.clear();
    }
    h->unet = n;
    h->unet_dirty = 1;
    return HICARW_OK;
}

// ---- the steps either side of the solve in update_winds (wind.F90) --------------
// Device pointers, caller (Fortran) layouts; stream-ordered, no host sync.
static int device_only(int mem_kind) { return mem_kind == HICARW_MEM_DEVICE ? 0 : HICARW_ERR_ARG; }

static int ensure_work(hicarw_handle *h)
{
    if (!h->swork) CK(cudaMalloc((void **)&h->swork, n_cell(h->d) * 4));
    return 0;
}

extern "C" int hicarw_calc_w_real(hicarw_handle *h, const float *u, const float *v, const float *w_grid, float *w_real,
                                  int mem_kind, void *stream)
{
    api_entry();
    if (!h || !u || !v || !w_real || device_only(mem_kind)) return HICARW_ERR_ARG;
    launch_w_real(h->d, metrics_of(h), u, v, w_grid, w_real, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_calc_idealized_wgrid(hicarw_handle *h, const float *u, const float *v, const float *w_real,
                                           float *w, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !u || !v || !w_real || !w || device_only(mem_kind)) return HICARW_ERR_ARG;
    launch_idealized_wgrid(h->d, metrics_of(h), u, v, w_real, w, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_balance_uvw(hicarw_handle *h, const float *u, const float *v, const float *density, float *w,
                                  int adv_den, int use_dqdt, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !u || !v || !w || (adv_den && !density) || device_only(mem_kind)) return HICARW_ERR_ARG;
    int rc;
    if ((rc = ensure_work(h)) != 0) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const Metrics m = metrics_of(h);
    launch_divergence(h->d, m, u, v, w, adv_den ? density : nullptr, h->swork, adv_den, 1, use_dqdt, s);
    launch_calc_w(h->d, m, h->swork, adv_den ? density : nullptr, w, adv_den, s);
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_calc_alpha(hicarw_handle *h, const float *froude, float *alpha, int halo, int mem_kind,
                                 void *stream)
{
    api_entry();
    if (!h || !froude || !alpha || halo < 0 || 2 * halo >= h->d.nx || 2 * halo >= h->d.ny || device_only(mem_kind))
        return HICARW_ERR_ARG;
    launch_calc_alpha(h->d, froude, alpha, halo, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return HICARW_OK;
}

// ---- decomposed solves (the reference's multi-rank BiCGStab, wind_iterative.F90:555-791 with
// exchange_krylov_halos :1552-1733 and the allreduces :604-729): the library computes, the
// caller communicates (NCCL, MPI or copies) between the steps ----
extern "C" int hicarw_dist_configure(hicarw_handle *h, int edges)
{
    api_entry();
    if (!h || edges < 0 || edges > 15) return HICARW_ERR_ARG;
    cudaDeviceSynchronize();
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
    h->graphs.clear();
    h->edges = edges;
    if (!h->dist_buf) CK(dalloc((void **)&h->dist_buf, 8 * sizeof(double)));
    return HICARW_OK;
}

static int dist_ready(hicarw_handle *h)
{
    if (!h || !h->dist_buf || h->opt.solver != HICARW_SOLVER_REFERENCE || h->opt.krylov_precision != HICARW_KRYLOV_F64)
        return HICARW_ERR_STATE;
    return 0;
}

// totals (device dist_tot) -> caller buffer
static int dist_out(hicarw_handle *h, double *tot, int n, int mem_kind, cudaStream_t s)
{
    CK(cudaMemcpyAsync(tot, h->st->dist_tot, n * sizeof(double),
                       mem_kind == HICARW_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    if (mem_kind == HICARW_MEM_HOST) CK(cudaStreamSynchronize(s));
    return 0;
}

extern "C" int hicarw_dist_setup(hicarw_handle *h, const double *rhs, double *tot3, int mem_kind, void *stream)
{
    api_entry();
    int rc;
    if ((rc = dist_ready(h)) != 0 || !rhs || !tot3) return rc ? rc : HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    select_precond(h, 1);
    if (h->use_learned || h->use_mglearned) return HICARW_ERR_STATE;
    if (h->use_mg && (h->mg_dirty || !h->mg.ready)) {
        mg_params(h);
        if (mg_build_tuned(h, s) != 0) return HICARW_ERR_CUDA;
        h->mg_dirty = 0;
    }
    if ((rc = ensure_vectors(h, HICARW_KRYLOV_F64)) != 0) return rc;
    if ((rc = put_padded(h, rhs, V<double>(h, V_RHS), mem_kind, s)) != 0) return rc;
    launch_diag<double>(h->d, h->coef, h->dz_if, V<double>(h, V_DINV), h->operator_probed, s);
    launch_zero_rank_edges<double>(h->d, h->edges, V<double>(h, V_DINV), s);
    launch_state_reset(h->st, h->opt.tol_rel, h->opt.tol_abs, h->opt.max_iters, 0, s);
    static const int one = 1;
    CK(cudaMemcpyAsync(&h->st->dist, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    OpCtx c = opctx(h);
    RedBuf rb{h->partials, h->red_blocks};
    enqueue_setup_prec(h, HICARW_KRYLOV_F64, c, rb, s, 0);
    CK(cudaGetLastError());
    return dist_out(h, tot3, 3, mem_kind, s);
}

extern "C" int hicarw_dist_apply(hicarw_handle *h, int kind, const double *tot, int mem_kind, void *stream)
{
    api_entry();
    int rc;
    if ((rc = dist_ready(h)) != 0) return rc;
    if (kind < 0 || kind > 2 || !tot) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = kind == 0 ? 3 : kind == 1 ? 1 : 5;
    const double *t = tot;
    if (mem_kind == HICARW_MEM_HOST) {
        CK(cudaMemcpyAsync(h->dist_buf, tot, n * sizeof(double), cudaMemcpyHostToDevice, s));
        t = h->dist_buf;
    }
    launch_dist_apply(h->st, h->hist, kind, t, s);
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_dist_precond(hicarw_handle *h, int which, void *stream)
{
    api_entry();
    int rc;
    if ((rc = dist_ready(h)) != 0) return rc;
    if (which < 0 || which > 1) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    SolveState *st = h->st;
    double *r = V<double>(h, V_R), *p = V<double>(h, V_P), *phat = V<double>(h, V_PHAT), *v = V<double>(h, V_V),
           *sv = V<double>(h, V_S), *shat = V<double>(h, V_SHAT), *Dinv = V<double>(h, V_DINV);
    if (which == 0) {
        launch_iteration_begin(st, s);
        if (h->use_mg) mg_apply<double>(h->mg, p, phat, st, s);
        else enqueue_precond<double>(h, p, phat, h->precond_n_sweeps, st, 0, s);
    } else if (h->use_mg) {
        launch_s_update<double>(h->d, r, v, sv, st, s);
        mg_apply<double>(h->mg, sv, shat, st, s);
    } else {
        OpCtx c = opctx(h);
        double *pres = V<double>(h, V_PRES);
        launch_s_precond<double>(h->d, r, v, sv, shat, Dinv, st, s);
        for (int sw = 2; sw <= h->precond_n_sweeps; sw++) {
            launch_spmv<double>(c, shat, pres, st, s);
            launch_rich<double>(h->d, sv, shat, pres, Dinv, st, s);
        }
    }
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_dist_face(hicarw_handle *h, int vec, int side, double *buf, int unpack, void *stream)
{
    api_entry();
    int rc;
    if ((rc = dist_ready(h)) != 0) return rc;
    if (vec < 0 || vec > 2 || side < 0 || side > 3 || !buf) return HICARW_ERR_ARG;
    const int q = vec == 0 ? V_PHAT : vec == 1 ? V_SHAT : V_X;
    launch_face(h->d, V<double>(h, q), side, buf, unpack != 0, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_dist_spmv(hicarw_handle *h, int which, double *tot, int mem_kind, void *stream)
{
    api_entry();
    int rc;
    if ((rc = dist_ready(h)) != 0) return rc;
    if (which < 0 || which > 1 || !tot) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    OpCtx c = opctx(h);
    RedBuf rb{h->partials, h->red_blocks};
    SolveState *st = h->st;
    double *rhat = V<double>(h, V_RHAT), *phat = V<double>(h, V_PHAT), *v = V<double>(h, V_V),
           *sv = V<double>(h, V_S), *shat = V<double>(h, V_SHAT), *t = V<double>(h, V_T);
    CK(cudaMemsetAsync(st->dist_tot, 0, 5 * sizeof(double), s)); // a solve that has stopped publishes zeros
    if (which == 0) launch_spmv_sigma<double>(c, phat, v, rhat, st, rb, s);
    else launch_spmv_dot5<double>(c, shat, t, sv, rhat, st, h->hist, rb, s);
    CK(cudaGetLastError());
    return dist_out(h, tot, which == 0 ? 1 : 5, mem_kind, s);
}

extern "C" int hicarw_dist_update(hicarw_handle *h, void *stream)
{
    api_entry();
    int rc;
    if ((rc = dist_ready(h)) != 0) return rc;
    double *x = V<double>(h, V_X), *r = V<double>(h, V_R), *p = V<double>(h, V_P), *phat = V<double>(h, V_PHAT),
           *v = V<double>(h, V_V), *sv = V<double>(h, V_S), *shat = V<double>(h, V_SHAT), *t = V<double>(h, V_T);
    launch_update_xrp<double, double>(h->d, x, phat, shat, r, sv, t, p, v, h->st, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_dist_state(hicarw_handle *h, int *stop, hicarw_stats *stats, void *stream)
{
    api_entry();
    int rc;
    if ((rc = dist_ready(h)) != 0) return rc;
    if ((rc = fetch_state(h, (cudaStream_t)stream)) != 0) return rc;
    if (stop) *stop = h->hst->stop;
    if (stats) fill_stats(h, stats, h->precond_n_sweeps, 0);
    return HICARW_OK;
}

extern "C" int hicarw_set_kernel_tuning(hicarw_handle *h, int spmv_levels, int mg_post_feed)
{
    api_entry();
    if (!h || spmv_levels < 0 || spmv_levels > 1024 || mg_post_feed < -1 || mg_post_feed > 1) return HICARW_ERR_ARG;
    cudaDeviceSynchronize();
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
    h->graphs.clear();
    h->tune_kc = spmv_levels;
    h->tune_mg_feed = mg_post_feed;
    if (mg_post_feed >= 0) h->mg.use_tma = mg_post_feed ? 2 : 0;
    else h->mg_dirty = 1; // the build decides again
    return HICARW_OK;
}

extern "C" int hicarw_debug_wait_timeout(hicarw_handle *h, double limit_us, void *stream)
{
    api_entry();
    if (!h || !(limit_us >= 1.0 && limit_us <= 100000.0)) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemsetAsync(&h->st->err, 0, sizeof(int), s));
    mg_wait_probe(&h->st->err, (uint64_t)(limit_us * 1000.0), s);
    CK(cudaGetLastError());
    const int rc = fetch_state(h, s); // HICARW_ERR_TIMEOUT when the wait gave up
    CK(cudaMemsetAsync(&h->st->err, 0, sizeof(int), s));
    CK(cudaStreamSynchronize(s));
    if (rc == HICARW_ERR_TIMEOUT) h->err = "a bounded device-side wait timed out (wait probe)";
    return rc;
}

extern "C" int hicarw_update_stability(hicarw_handle *h, const float *u, const float *v, const float *z,
                                       const float *theta, const float *froude_terrain, int nsect, int froude_mode,
                                       float *froude, float *blk_ri, int mem_kind, void *stream)
{
    api_entry();
    if (!h || !u || !v || !z || !theta || !froude || !blk_ri || h->d.nz < 5 || device_only(mem_kind) ||
        (froude_mode && (!froude_terrain || nsect < 1)))
        return HICARW_ERR_ARG;
    launch_update_stability(h->d, u, v, z, theta, froude_terrain, nsect, froude_mode, froude, blk_ri,
                            (cudaStream_t)stream);
    CK(cudaGetLastError());
    return HICARW_OK;
}

extern "C" int hicarw_smooth_alpha(hicarw_handle *h, float *alpha, int window, int nsmooths, int mem_kind,
                                   void *stream)
{
    api_entry();
    if (!h || !alpha || window < 0 || nsmooths < 0 || device_only(mem_kind)) return HICARW_ERR_ARG;
    int rc;
    if ((rc = ensure_work(h)) != 0) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    for (int p = 0; p < nsmooths; p++) {
        CK(cudaMemcpyAsync(h->swork, alpha, n_cell(h->d) * 4, cudaMemcpyDeviceToDevice, s));
        launch_smooth_xy(h->d, h->swork, alpha, window, s);
    }
    CK(cudaGetLastError());
    return HICARW_OK;
}

// ---- batched solves of independent subdomains ---------------------------------
// One CUDA graph solves every subdomain of the batch: per subdomain a chain
// [inputs + RHS + BiCGStab set-up] -> WHILE node whose body is `chunk`
// iterations plus a one-thread kernel that keeps the loop running while the
// device-side solve state has not stopped.  So a whole batch of uneven solves
// is one graph launch and one host synchronisation; the subdomains are spread
// over `lanes` independent chains (longest-processing-time order by size) that
// the GPU runs concurrently.  Every WHILE loop is also bounded by a body count
// (max_iters / chunk + 2), so it ends even if a solve never sets its flag.
// a failed batch call: the message is the one hicarw_last_error(NULL) returns
static int batch_fail(int rc, const std::string &msg)
{
    g_err_noh = "hicarw batch: " + msg;
    fprintf(stderr, "%s\n", g_err_noh.c_str());
    return rc;
}

#define BCK(x)                                                                                                   \
    do {                                                                                                         \
        cudaError_t e_ = (x);                                                                                    \
        if (e_ != cudaSuccess) return batch_fail(HICARW_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct hicarw_batch {
    std::vector<hicarw_handle *> hs;
    int lanes = 0, chunk = 4; // lanes <= 0: one chain per subdomain
    cudaGraphExec_t exec = nullptr;
    long long nodes = 0;
    std::vector<hicarw_batch_item> built;
    int built_lanes = -1, built_chunk = -1, built_cold = -1;
    std::vector<FgmresCtx> fg; // launch contexts of the FGMRES subdomains
    int *counters = nullptr; // device: WHILE-body executions per subdomain
    unsigned long long *stamps = nullptr; // device: %globaltimer at each solve's end, [n] = batch start
    cudaStream_t cap = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    float last_ms = 0.0f;
};

__global__ void batch_count_reset_kernel(int *count) { *count = 0; }

__global__ void batch_stamp_kernel(unsigned long long *slot)
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *slot = t;
}

// a child-graph node holding one timestamp kernel
static cudaError_t batch_stamp_node(hicarw_batch *b, cudaGraph_t g, const cudaGraphNode_t *dep, int ndep,
                                    unsigned long long *slot, cudaGraphNode_t *out)
{
    cudaGraph_t sg;
    cudaError_t e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    batch_stamp_kernel<<<1, 1, 0, b->cap>>>(slot);
    count_launch(1);
    e = cudaStreamEndCapture(b->cap, &sg);
    if (e != cudaSuccess) return e;
    e = cudaGraphAddChildGraphNode(out, g, dep, ndep, sg);
    cudaGraphDestroy(sg);
    return e;
}

// FGMRES subdomains loop over restart cycles until converged or out of iterations
__global__ void batch_fg_cond_kernel(cudaGraphConditionalHandle hc, const GmresState *g, int *count, int limit)
{
    const int c = *count + 1;
    *count = c;
    const int more = g->status != 0 && g->it_total < g->max_iters && c < limit;
    cudaGraphSetConditional(hc, more ? 1u : 0u);
}

__global__ void batch_cond_kernel(cudaGraphConditionalHandle hc, const SolveState *st, int *count, int limit)
{
    const int c = *count + 1;
    *count = c;
    const int more = !*(volatile const int *)&st->stop && c < limit;
    cudaGraphSetConditional(hc, more ? 1u : 0u);
}

static bool same_items(const hicarw_batch *b, const hicarw_batch_item *items)
{
    if (b->built.size() != b->hs.size()) return false;
    for (size_t i = 0; i < b->hs.size(); i++) {
        const hicarw_batch_item &x = b->built[i], &y = items[i];
        if (x.alpha != y.alpha || x.div != y.div || x.density != y.density || x.u != y.u || x.v != y.v || x.w != y.w)
            return false;
    }
    return true;
}

static void batch_drop_graph(hicarw_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->built.clear();
}

// enqueue (capture) the per-subdomain set-up: inputs, diagonal, RHS, solve state, r = b - A x
static void batch_enqueue_setup(hicarw_batch *b, int i, const hicarw_batch_item &it, int cold, cudaStream_t s)
{
    hicarw_handle *h = b->hs[i];
    const Dims &d = h->d;
    cudaMemcpyAsync(h->alpha, it.alpha, n_cell(d) * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(h->div, it.div, n_cell(d) * 4, cudaMemcpyDeviceToDevice, s);
    if (cold) cudaMemsetAsync(h->vec[V_X], 0, (size_t)d.npad * 8, s);
    prepare_system(h, s);
    if (h->opt.solver == HICARW_SOLVER_FGMRES) {
        fgmres_reset(h->gst, b->fg[i].m, h->opt.tol_rel, h->opt.tol_abs, h->opt.max_iters, h->hist, h->st, s);
    } else {
        launch_state_reset(h->st, h->opt.tol_rel, h->opt.tol_abs, h->opt.max_iters, h->use_mg ? h->opt.stall_iters : 0,
                           s);
        OpCtx c = opctx(h);
        RedBuf rb{h->partials, h->red_blocks};
        launch_setup<double, double>(c, V<double>(h, V_X), V<double>(h, V_RHS), V<double>(h, V_R),
                                     V<double>(h, V_RHAT), V<double>(h, V_P), h->st, h->hist, rb, 0, s);
    }
    batch_count_reset_kernel<<<1, 1, 0, s>>>(b->counters + i);
    count_launch(1);
}

static int batch_build(hicarw_batch *b, const hicarw_batch_item *items, int cold)
{
    batch_drop_graph(b);
    const int n = (int)b->hs.size();
    const int lanes = b->lanes <= 0 || b->lanes > n ? n : b->lanes;
    // longest processing time first: biggest subdomain to the least loaded lane
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int c) { return b->hs[a]->d.npad > b->hs[c]->d.npad; });
    std::vector<long long> load(lanes, 0);
    std::vector<cudaGraphNode_t> tail(lanes, nullptr);
    cudaGraph_t g;
    BCK(cudaGraphCreate(&g, 0));
    long long nodes = 0;
    cudaGraphNode_t root;
    cudaError_t e = batch_stamp_node(b, g, nullptr, 0, b->stamps + n, &root);
    for (int L = 0; L < lanes; L++) tail[L] = root;
    for (int oi = 0; oi < n && e == cudaSuccess; oi++) {
        const int i = order[oi];
        hicarw_handle *h = b->hs[i];
        int L = 0;
        for (int q = 1; q < lanes; q++)
            if (load[q] < load[L]) L = q;
        load[L] += h->d.npad;
        // set-up as a child graph
        cudaGraph_t sg;
        g_capturing = 1;
        g_capture_nodes = 0;
        e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) break;
        batch_enqueue_setup(b, i, items[i], cold, b->cap);
        e = cudaStreamEndCapture(b->cap, &sg);
        g_capturing = 0;
        if (e != cudaSuccess) break;
        nodes += g_capture_nodes;
        cudaGraphNode_t sn, wn;
        e = cudaGraphAddChildGraphNode(&sn, g, &tail[L], 1, sg);
        cudaGraphDestroy(sg);
        if (e != cudaSuccess) break;
        // the device-driven loop
        cudaGraphConditionalHandle hc;
        e = cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) break;
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = hc;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        e = cudaGraphAddNode(&wn, g, &sn, 1, &p);
        if (e != cudaSuccess) break;
        cudaGraph_t body = p.conditional.phGraph_out[0];
        g_capturing = 1;
        g_capture_nodes = 0;
        e = cudaStreamBeginCaptureToGraph(b->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { g_capturing = 0; break; }
        if (h->opt.solver == HICARW_SOLVER_FGMRES) { // body: one restart cycle
            fgmres_enqueue_cycle(b->fg[i], b->cap);
            batch_fg_cond_kernel<<<1, 1, 0, b->cap>>>(hc, h->gst, b->counters + i, h->opt.max_iters / b->fg[i].m + 2);
        } else {
            for (int q = 0; q < b->chunk; q++)
                enqueue_iteration<double, double>(h, V<double>(h, V_X), h->precond_n_sweeps, b->cap);
            batch_cond_kernel<<<1, 1, 0, b->cap>>>(hc, h->st, b->counters + i, h->opt.max_iters / b->chunk + 2);
        }
        count_launch(1);
        e = cudaStreamEndCapture(b->cap, &body);
        g_capturing = 0;
        nodes += g_capture_nodes;
        if (e != cudaSuccess) break;
        cudaGraphNode_t tn;
        e = batch_stamp_node(b, g, &wn, 1, b->stamps + i, &tn);
        tail[L] = tn;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->exec = nullptr;
        return batch_fail(HICARW_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
    }
    b->nodes = nodes;
    b->built.assign(items, items + n);
    b->built_lanes = b->lanes;
    b->built_chunk = b->chunk;
    b->built_cold = cold;
    return 0;
}

// One batched solve; apply != 0 also corrects the winds.  stats: n entries or null.
static int batch_run(hicarw_batch *b, const hicarw_batch_item *items, int adv_den, int cold, int apply, cudaStream_t s,
                     hicarw_stats *stats)
{
    const int n = (int)b->hs.size();
    int rc;
    bool rebuild = !b->exec || !same_items(b, items) || b->built_lanes != b->lanes || b->built_chunk != b->chunk ||
                   b->built_cold != cold;
    b->fg.resize(n);
    for (int i = 0; i < n; i++) {
        hicarw_handle *h = b->hs[i];
        h->launches_at_call = g_launches.load();
        select_precond(h, 1);
        if (h->use_mg && (h->mg_dirty || !h->mg.ready)) {
            mg_params(h);
            if (mg_build_tuned(h, s) != 0)
                return batch_fail(HICARW_ERR_CUDA, "multigrid build of subdomain " + std::to_string(i) + ": " + h->err);
            h->mg_dirty = 0;
            rebuild = true;
        }
        if (h->opt.solver == HICARW_SOLVER_FGMRES) {
            const bool dirty = (h->use_learned || h->use_mglearned) && h->unet_dirty;
            FgmresCtx f;
            if ((rc = fgmres_ready(h, h->precond_n_sweeps, s, &f)) != 0)
                return batch_fail(rc, "FGMRES set-up of subdomain " + std::to_string(i) + ": " + h->err);
            if (dirty || b->fg[i].V != f.V || b->fg[i].m != f.m) rebuild = true;
            b->fg[i] = f;
        }
    }
    if (rebuild) {
        BCK(cudaStreamSynchronize(s));
        if ((rc = batch_build(b, items, cold)) != 0) return rc;
    }
    BCK(cudaEventRecord(b->t0, s));
    for (int i = 0; i < n; i++) BCK(cudaEventRecord(b->hs[i]->t0, s)); // per-handle solve time = the batch's
    BCK(cudaGraphLaunch(b->exec, s));
    g_launches += b->nodes;
    BCK(cudaEventRecord(b->t1, s));
    for (int i = 0; i < n; i++) BCK(cudaEventRecord(b->hs[i]->t1, s));
    for (int i = 0; i < n; i++)
        BCK(cudaMemcpyAsync(b->hs[i]->hst, b->hs[i]->st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    BCK(cudaEventElapsedTime(&b->last_ms, b->t0, b->t1));
    for (int i = 0; i < n; i++)
        if (b->hs[i]->hst->err)
            return batch_fail(HICARW_ERR_TIMEOUT, "subdomain " + std::to_string(i) + ": a bounded device-side wait timed out");
    for (int i = 0; i < n; i++) // FGMRES state -> the solve-state mirror
        if (b->hs[i]->opt.solver == HICARW_SOLVER_FGMRES && (rc = fgmres_map_state(b->hs[i], 0, s)) != 0)
            return batch_fail(rc, "FGMRES state of subdomain " + std::to_string(i) + ": " + b->hs[i]->err);
    std::vector<int> fell(n, 0);
    for (int i = 0; i < n; i++) { // a stalled or failed preconditioned solve: the reference solve decides
        hicarw_handle *h = b->hs[i];
        if (h->hst->status != 0 && (h->use_mg || h->use_learned)) {
            if ((rc = zero_solution(h, s)) != 0 || (rc = bicgstab_solve(h, h->precond_n_sweeps, s, 0)) != 0)
                return batch_fail(rc, "fallback solve of subdomain " + std::to_string(i) + ": " + h->err);
            fell[i] = 1;
        }
    }
    for (int i = 0; i < n; i++) {
        hicarw_handle *h = b->hs[i];
        OpCtx c = opctx(h);
        RedBuf rb{h->partials, h->red_blocks};
        if (h->opt.solver != HICARW_SOLVER_FGMRES || fell[i])
            launch_true_residual<double, double>(c, V<double>(h, V_X), V<double>(h, V_RHS), nullptr, nullptr, h->st, 0,
                                                 rb, s);
        if (apply) enqueue_winds(h, adv_den ? items[i].density : nullptr, adv_den, items[i].u, items[i].v, items[i].w, s);
        if (h->opt.solver != HICARW_SOLVER_FGMRES || fell[i]) // FGMRES stats were mapped above
            BCK(cudaMemcpyAsync(h->hst, h->st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
    }
    BCK(cudaStreamSynchronize(s));
    if (stats)
        for (int i = 0; i < n; i++) {
            fill_stats(b->hs[i], &stats[i], b->hs[i]->precond_n_sweeps, 0);
            stats[i].solve_ms = b->last_ms;
            if (fell[i]) {
                stats[i].status = HICARW_FELL_BACK;
                stats[i].precond = HICARW_PRECOND_JACOBI;
            }
        }
    return HICARW_OK;
}

extern "C" int hicarw_batch_create(int n, hicarw_handle *const *handles, hicarw_batch **out)
{
    api_entry();
    if (n < 1 || !handles || !out) return HICARW_ERR_ARG;
    for (int i = 0; i < n; i++) {
        hicarw_handle *h = handles[i];
        const bool bicg = h && h->opt.solver == HICARW_SOLVER_REFERENCE && h->opt.krylov_precision == HICARW_KRYLOV_F64;
        const bool fgm = h && h->opt.solver == HICARW_SOLVER_FGMRES;
        if (!h || !h->operator_probed || !(bicg || fgm))
            return HICARW_ERR_ARG; // calibrated handles: FP64 BiCGStab (reference schedule) or FGMRES
        for (int q = 0; q < i; q++)
            if (handles[q] == h) return HICARW_ERR_ARG;
        if (ensure_vectors(h, HICARW_KRYLOV_F64) != 0) return HICARW_ERR_CUDA;
    }
    hicarw_batch *b = new hicarw_batch();
    b->hs.assign(handles, handles + n);
    if (cudaMalloc((void **)&b->counters, n * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&b->stamps, (n + 1) * sizeof(unsigned long long)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->t0) != cudaSuccess || cudaEventCreate(&b->t1) != cudaSuccess) {
        delete b;
        return HICARW_ERR_CUDA;
    }
    cudaMemset(b->counters, 0, n * sizeof(int));
    *out = b;
    return HICARW_OK;
}

extern "C" int hicarw_batch_destroy(hicarw_batch *b)
{
    api_entry();
    if (!b) return HICARW_ERR_ARG;
    cudaDeviceSynchronize();
    batch_drop_graph(b);
    if (b->counters) cudaFree(b->counters);
    if (b->stamps) cudaFree(b->stamps);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->t1) cudaEventDestroy(b->t1);
    delete b;
    return HICARW_OK;
}

extern "C" int hicarw_batch_config(hicarw_batch *b, int lanes, int chunk)
{
    api_entry();
    if (!b || chunk < 1 || chunk > 64) return HICARW_ERR_ARG;
    b->lanes = lanes;
    b->chunk = chunk;
    return HICARW_OK;
}

extern "C" int hicarw_batch_get_config(const hicarw_batch *b, int *lanes, int *chunk)
{
    api_entry();
    if (!b) return HICARW_ERR_ARG;
    if (lanes) *lanes = b->lanes <= 0 ? (int)b->hs.size() : b->lanes;
    if (chunk) *chunk = b->chunk;
    return HICARW_OK;
}

extern "C" int hicarw_batch_calc_iter_winds(hicarw_batch *b, const hicarw_batch_item *items, int adv_den, int cold,
                                            void *stream, hicarw_stats *stats)
{
    api_entry();
    if (!b || !items) return HICARW_ERR_ARG;
    for (size_t i = 0; i < b->hs.size(); i++)
        if (!items[i].alpha || !items[i].div || !items[i].u || !items[i].v || !items[i].w ||
            (adv_den && !items[i].density))
            return HICARW_ERR_ARG;
    return batch_run(b, items, adv_den, cold, 1, (cudaStream_t)stream, stats);
}

// Per-subdomain solve latency of the last batched call: milliseconds from the
// start of the batch graph to the end of that subdomain's solve loop.
extern "C" int hicarw_batch_latencies(hicarw_batch *b, double *ms)
{
    api_entry();
    if (!b || !ms || !b->exec) return HICARW_ERR_ARG;
    const int n = (int)b->hs.size();
    std::vector<unsigned long long> t(n + 1);
    BCK(cudaMemcpy(t.data(), b->stamps, (n + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) ms[i] = t[i] >= t[n] ? (double)(t[i] - t[n]) * 1e-6 : 0.0;
    return HICARW_OK;
}

// Autotuner: time cold batched solves (no wind correction) for every (lanes,
// chunk) candidate and keep the fastest; the solutions are cleared afterwards.
extern "C" int hicarw_batch_autotune(hicarw_batch *b, const hicarw_batch_item *items, int adv_den, void *stream,
                                     double *best_ms)
{
    api_entry();
    if (!b || !items) return HICARW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = (int)b->hs.size();
    const int lane_c[] = {1, 4, 16, 64};
    const int chunk_c[] = {4, 8};
    double best = 1e300;
    int bl = b->lanes, bc = b->chunk;
    for (int lc : lane_c) {
        if (lc > n) continue;
        for (int cc : chunk_c) {
            b->lanes = lc;
            b->chunk = cc;
            int rc = batch_run(b, items, adv_den, 1, 0, s, nullptr); // build + warm
            if (rc) return rc;
            if ((rc = batch_run(b, items, adv_den, 1, 0, s, nullptr)) != 0) return rc;
            if (b->last_ms < best) {
                best = b->last_ms;
                bl = lc;
                bc = cc;
            }
        }
    }
    b->lanes = bl;
    b->chunk = bc;
    batch_drop_graph(b);
    for (int i = 0; i < n; i++) zero_solution(b->hs[i], s);
    BCK(cudaStreamSynchronize(s));
    if (best_ms) *best_ms = best;
    return HICARW_OK;
}

// ---- accessors for the entry points defined in other files ----
namespace hw {
void handle_operator(const hicarw_handle *h, OpCtx *c) { *c = opctx(h); }
void handle_set_error(hicarw_handle *h, const char *msg) { h->err = msg; }
}  // namespace hw

