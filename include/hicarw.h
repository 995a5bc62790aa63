/*
 * hicarw.h -- C ABI of the B200 iterative wind solver.
 *
 * Drop-in replacement for HICAR's Fortran module `wind_iterative`
 * (src/physics/wind_iterative.F90).  Each entry point below names the
 * reference routine it replaces.  The Fortran side binds these functions
 * with ISO_C_BINDING (bind(C) interfaces); every argument is a plain pointer,
 * an int or a float/double, every array uses the reference's Fortran layout
 * (i fastest, then k, then j), and every function returns an int status:
 *
 *     0  HICARW_OK                 converged / done
 *     1  HICARW_ITER_CAP           iteration cap reached (reference status 1)
 *     2  HICARW_BREAKDOWN          BiCGStab breakdown (reference status 2)
 *     3  HICARW_FELL_BACK          flexible/learned solve fell back to plain BiCGStab
 *    <0  an error (argument, state, CUDA, or the reference's fatal `stop`);
 *        the library never aborts the caller.
 *
 * Array pointers are device pointers (mem_kind = HICARW_MEM_DEVICE, e.g. an
 * OpenACC `host_data use_device` region) or host pointers
 * (HICARW_MEM_HOST: the library stages them through its own device buffers).
 * Work is ordered on the CUDA stream passed in (NULL = legacy default stream);
 * entry points return after the work is enqueued unless they hand a result
 * back to host memory (stats, leakage), in which case they synchronise the stream.
 *
 * Threading: one handle per nest; a handle is not thread-safe.
 *
 * Array extents at one rank (nx = ide, ny = jde, nz = kde):
 *   cell     (nx, nz, ny)     alpha, div, density, jacobian, jacobian_w, dzdx,
 *                             dzdy, advection_dz, w (w%dqdt_3d)
 *   u-face   (nx+1, nz, ny)   u (u%dqdt_3d), jacobian_u, dzdx_u
 *   v-face   (nx, nz, ny+1)   v (v%dqdt_3d), jacobian_v, dzdy_v
 *   2-D      (nx, ny)         neighbor_terrain, mapfac_mxy
 *            (nx+1, ny)       mapfac_mx_u, mapfac_my_u
 *            (nx, ny+1)       mapfac_my_v, mapfac_mx_v
 */
#ifndef HICARW_H
#define HICARW_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HICARW_ABI_VERSION 2

enum {
    HICARW_OK = 0,
    HICARW_ITER_CAP = 1,
    HICARW_BREAKDOWN = 2,
    HICARW_FELL_BACK = 3,
    HICARW_ERR_ARG = -1,
    HICARW_ERR_STATE = -2,
    HICARW_ERR_CUDA = -3,
    HICARW_ERR_DIVERGED = -4, /* the reference executes `stop` here (wind_iterative.F90:506-528) */
    HICARW_ERR_NAN = -5,
    HICARW_ERR_TIMEOUT = -6   /* a bounded device-side wait gave up */
};

enum { HICARW_MEM_DEVICE = 0, HICARW_MEM_HOST = 1 };

/* Krylov vector precision. */
enum {
    HICARW_KRYLOV_F64 = 0,    /* reference precision: FP64 vectors, FP64 reductions */
    HICARW_KRYLOV_F32 = 1,    /* withdrawn (FP32 vectors and FP32 lambda: the solution drifts, and the
                                 schedule diverged at 512x512x48): rejected with HICARW_ERR_ARG */
    HICARW_KRYLOV_F32_X64 = 2 /* FP32 vectors, FP64 reductions and FP64 accumulation of lambda (the
                                 solution): the true residual follows the recurrence residual (reference
                                 schedule) */
};

/* Solve schedule. */
enum {
    HICARW_SOLVER_REFERENCE = 0, /* right-preconditioned BiCGStab, reference kernel schedule */
    HICARW_SOLVER_FUSED = 1,     /* withdrawn (the fused FP32 schedule): rejected with HICARW_ERR_ARG */
    HICARW_SOLVER_MIXED = 2,     /* shorthand: the reference schedule with HICARW_KRYLOV_F32_X64 and
                                    HICARW_CRIT_TRUE (FP32 vectors, FP64 reductions and lambda, periodic
                                    FP64 residual replacement, restarts until the FP64 true residual
                                    meets the target: iterative refinement of lambda) */
    HICARW_SOLVER_FGMRES = 3     /* flexible GMRES(m), FP64 Krylov, right-preconditioned with any
                                    (also variable) preconditioner; the outer loop of the learned one */
};

/* Preconditioner. */
enum {
    HICARW_PRECOND_JACOBI = 0, /* the reference's Block-Jacobi / Jacobi-Richardson sweeps (:1268-1315) */
    HICARW_PRECOND_MG = 1,     /* multigrid V-cycle: z-line Jacobi smoother, 2x2 x-y aggregation,
                                  Galerkin coarse operators down to one column (probed operator only) */
    HICARW_PRECOND_LEARNED = 2, /* the U-Net attached by hicarw_set_learned_precond (FGMRES only,
                                   probed operator only) */
    HICARW_PRECOND_MG_LEARNED = 3 /* the V-cycle, then the attached U-Net's correction u = U(r') of the
                                     residual r' = r - A M(r) it leaves, taken with the minimal-residual step:
                                     z = M(r) + theta u, theta = <r', A u> / <A u, A u>, so ||r - A z|| <= ||r'||
                                     (FGMRES only, probed operator only) */
};

/* Stopping rule. */
enum {
    HICARW_CRIT_RECURRENCE = 0, /* ||s - w t|| <= max(tol_abs, tol_rel ||b||) (wind_iterative.F90:633,758) */
    HICARW_CRIT_TRUE = 1        /* additionally ||b - A x|| (FP64) <= max(tol_abs, tol_rel ||b||): while it is
                                   not, the BiCGStab recurrences restart from the current solution */
};

typedef struct hicarw_grid {
    int nx, ny, nz; /* ide, jde, kde at one rank */
    float dx;       /* domain%dx */
    int nest;       /* domain%nest_indx (1..4) */
} hicarw_grid;

typedef struct hicarw_options {
    int max_iters;        /* wind%wind_solver_iterations (default 1500) */
    int verbose;          /* general%debug .or. windtype == kITERATIVE_WINDS */
    double tol_rel;       /* reference: 1e-5 (wind_iterative.F90:60) */
    double tol_abs;       /* reference: 1e-10 (wind_iterative.F90:59) */
    int krylov_precision; /* HICARW_KRYLOV_* */
    int solver;           /* HICARW_SOLVER_* */
    int criterion;        /* HICARW_CRIT_* */
    int replace_every;    /* FP32 Krylov vectors: the recurrence residual is replaced by the FP64 true
                             residual b - A x every replace_every iterations (rounded down to a multiple
                             of check_every; default 50) */
    int check_every;      /* iterations between host reads of the device-side stop flag */
    int precond;          /* HICARW_PRECOND_* */
    int stall_iters;      /* stop a preconditioned solve whose residual has not dropped by 1% for
                             this many iterations and fall back to the reference solve (0 = off) */
    float mg_omega;       /* damping of the multigrid smoother (default 0.8) */
    int fgmres_restart;   /* FGMRES restart length m (1..32, default 30) */
    float mg_coarse_scale; /* V-cycle: scale of the prolongated coarse-grid correction; over-correction
                              of the piecewise-constant aggregation (default 1.35) */
    int mg_skip_fine_presmooth; /* V-cycle: 0 = pre-smooth the finest level (default); 1 = restrict the
                                   right-hand side directly there (V(0,1) on the finest level: one
                                   smoother and one operator pass fewer per cycle) */
    int mg_w_levels;      /* V-cycle: bit l (l >= 1) makes level l correct twice from its coarse grid
                             (a W-cycle on those levels; bit 0 is ignored); 0 = V-cycle (default) */
    int mg_precision;     /* V-cycle coefficient storage: 0 = FP32 (default); 1 = BF16 for the finest level's
                             post-smoother (with mg_skip_fine_presmooth = 1, the only kernel that reads them;
                             its Thomas factors are those of the BF16-rounded tridiagonal; FP32 arithmetic) */
} hicarw_options;

/* Domain fields the solver reads (domain%vars_3d / vars_2d / mapfac_*),
 * wind_iterative.F90:2320-2331 and wind.F90:272-287. */
typedef struct hicarw_metrics {
    const float *jacobian, *jacobian_u, *jacobian_v, *jacobian_w;
    const float *dzdx, *dzdy, *dzdx_u, *dzdy_v;
    const float *advection_dz;
    const float *neighbor_terrain;
    const float *mapfac_mx_u, *mapfac_my_v, *mapfac_my_u, *mapfac_mx_v, *mapfac_mxy;
} hicarw_metrics;

typedef struct hicarw_stats {
    int status;        /* 0 converged, 1 iteration cap, 2 breakdown, 3 fell back, 4 stalled */
    int iterations;    /* BiCGStab iterations of the accepted solve */
    int sweeps;        /* Jacobi-Richardson sweeps of the accepted solve */
    int retries;       /* adaptive sweep retries (wind_iterative.F90:479-503) */
    double res0;       /* ||r0|| */
    double res_final;  /* recurrence norm at exit */
    double b_norm;     /* ||b|| */
    double target;     /* max(tol_abs, tol_rel ||b||) */
    double true_res;   /* ||b - A x|| in FP64 at exit (negative when not computed) */
    int replacements;  /* FP64 residual replacements and restarts (FP32 Krylov vectors) */
    int launches;      /* kernels launched by this call (incl. graph nodes) */
    int precond;       /* preconditioner of the accepted solve */
    double solve_ms;   /* device time of the Krylov solve (CUDA events) */
} hicarw_stats;

typedef struct hicarw_handle hicarw_handle;
typedef struct hicarw_unet hicarw_unet;
typedef struct hicarw_batch hicarw_batch;

/* Default options: the reference's constants (max_iters 1500, tol 1e-5/1e-10,
 * FP64 Krylov vectors, reference schedule, recurrence-norm stop). */
void hicarw_default_options(hicarw_options *opt);

/* init_iter_winds(domain, options)  (wind_iterative.F90:215-287, init_module_vars :2274-2421).
 * Copies the metric fields to device-resident solver state (one handle per nest,
 * the analogue of the reference's per-nest cache, :2613-2851). */
int hicarw_init_iter_winds(const hicarw_grid *grid, const hicarw_options *opt, const hicarw_metrics *m,
                           int mem_kind, void *stream, hicarw_handle **out);

/* finalize_iter_winds()  (wind_iterative.F90:2142-2267). Frees every device allocation. */
int hicarw_finalize_iter_winds(hicarw_handle *h);

/* calc_iter_winds(domain, alpha_in, div_in, adv_den)  (wind_iterative.F90:295-532):
 * first call builds the analytic coefficients (:351-407), later calls refresh them
 * when alpha varies and the operator is not probed (:408-427); then the diagonal,
 * the RHS b = -2 div, the warm-started BiCGStab solve with the adaptive sweep retry,
 * and the lambda -> (u, v, w_grid) correction (calc_updated_winds, :1742-2071)
 * applied in place to u, v, w (u%dqdt_3d, v%dqdt_3d, w%dqdt_3d).
 * density is domain%vars_3d(density); it is read only when adv_den != 0. */
int hicarw_calc_iter_winds(hicarw_handle *h, const float *alpha, const float *div, const float *density,
                           int adv_den, float *u, float *v, float *w, int mem_kind, void *stream,
                           hicarw_stats *stats);

/* calc_divergence(div, domain, advect_density, horz_only, use_dqdt)  (wind.F90:250-523). */
int hicarw_calc_divergence(hicarw_handle *h, const float *u, const float *v, const float *w,
                           const float *density, float *div, int adv_den, int horz_only, int use_dqdt,
                           int mem_kind, void *stream);

/* Probe hooks (wind_iterative.F90:1096-1248), called in this order for each of
 * the 27 colourings by calibrate_projection_operator (wind.F90:1055-1067). */
int hicarw_probe_lambda_pattern(hicarw_handle *h, int ca, int cb, int cc, void *stream);               /* :1096-1115 */
int hicarw_probe_zero_corrections(hicarw_handle *h, float *u, float *v, float *w, int mem_kind,
                                  void *stream);                                                       /* :1119-1155 */
int hicarw_probe_apply_corrections(hicarw_handle *h, const float *alpha, const float *density,
                                   int adv_den, float *u, float *v, float *w, int mem_kind,
                                   void *stream);                                                      /* :1158-1163 */
int hicarw_probe_record(hicarw_handle *h, const float *Tfield, int ca, int cb, int cc,
                        float *max_leak, int mem_kind, void *stream);                                 /* :1169-1231 */
int hicarw_probe_finalize(hicarw_handle *h, float max_leak, void *stream);                              /* :1235-1248 */

/* calibrate_projection_operator(domain, options, div)  (wind.F90:1010-1099):
 * all 27 probes on the device, no host round trip; u, v, w are used as scratch
 * and restored, as the reference does. */
int hicarw_calibrate_projection_operator(hicarw_handle *h, const float *alpha, const float *density,
                                         int adv_den, float *u, float *v, float *w, float *max_leak,
                                         int mem_kind, void *stream);

/* ---- extensions with no entry point of their own in the reference ---- */

/* Reset the warm-start lambda (x_sol) to zero, as probe_finalize does (:1243). */
int hicarw_reset_solution(hicarw_handle *h, void *stream);

/* Copy lambda (x_sol, FP64, (nx+2, nz+2, ny+2) Fortran layout) to the caller. */
int hicarw_get_lambda(hicarw_handle *h, double *lambda, int mem_kind, void *stream);

/* Copy the 15 stencil coefficients A..O ((nx, nz, ny) each, 15 consecutive arrays). */
int hicarw_get_coefs(hicarw_handle *h, float *coefs, int mem_kind, void *stream);
int hicarw_set_coefs(hicarw_handle *h, const float *coefs, int probed, int mem_kind, void *stream);

/* y = A x over all rows (spmv, wind_iterative.F90:813-1027); x, y FP64 (nx+2, nz+2, ny+2). */
int hicarw_apply_operator(hicarw_handle *h, const double *x, double *y, int mem_kind, void *stream);

/* y = M^-1 x: sweeps >= 1 applies the reference preconditioner (apply_precond,
 * wind_iterative.F90:1268-1315) with that many sweeps; sweeps == 0 applies one
 * multigrid V-cycle (probed operator only); sweeps < 0 applies the learned
 * preconditioner the options name (HICARW_PRECOND_LEARNED or _MG_LEARNED, with
 * the attached U-Net), else the V-cycle. */
int hicarw_apply_precond(hicarw_handle *h, const double *x, double *y, int sweeps, int mem_kind, void *stream);

/* Solve A lambda = rhs for a caller-given right-hand side ((nx+2, nz+2, ny+2), FP64),
 * starting from the current lambda; used by manufactured-solution tests. */
int hicarw_solve_rhs(hicarw_handle *h, const double *rhs, int mem_kind, void *stream, hicarw_stats *stats);

/* Change the solve options of an existing handle (precision, schedule, tolerance). */
int hicarw_set_options(hicarw_handle *h, const hicarw_options *opt);

/* Recurrence residual norm per iteration of the last solve (FP64). Returns the count. */
int hicarw_get_history(hicarw_handle *h, double *out, int cap);

/* Profile one solve iteration of the current configuration: every kernel of the
 * iteration is launched on its own `reps` times and timed with CUDA events on
 * `stream`.  For each distinct kernel (first-launch order, at most cap): its
 * name (32 bytes each in names), mean duration in ms, mean algorithmic bytes
 * of one launch, and launches per iteration.  With HICARW_SOLVER_FGMRES one
 * iteration is one restart cycle (fgmres_restart Arnoldi steps).  Returns the
 * number of kernels.  The solution is reset to zero. */
int hicarw_profile_iteration(hicarw_handle *h, int reps, char *names, double *ms, double *bytes, int *per_iter,
                             int cap, void *stream);

/* ||rhs - A x||_2 in FP64 for the handle's current operator, written to the
 * device double *norm; x and rhs are device arrays in the (nx+2, nz+2, ny+2)
 * Fortran layout.  This entry point has no counterpart in the reference.  It
 * allocates nothing, for callers that cannot call cudaMalloc (inside a stream
 * capture, or in a host model whose device memory is fixed up front): its
 * scratch is a static device array of 8192 FP64 plane partials, so ny + 2 <=
 * 8192 (larger grids return HICARW_ERR_ARG).  The first call on a device looks
 * up that array's address and should come before any stream capture; calls
 * that overlap on the GPU race on the shared array. */
int hicarw_residual_norm_noalloc(hicarw_handle *h, const double *x, const double *rhs, double *norm, void *stream);

/* ---- decomposed solves over several ranks (GPUs) ----
 * The reference's multi-rank BiCGStab (bicgstab_solve, wind_iterative.F90:555-791,
 * with exchange_krylov_halos :1552-1733 and the FP64 allreduces of 3, 1 and 5
 * values :604-729), split at its communication points: the library computes,
 * the caller communicates (NCCL send/recv and allreduce into its own device
 * buffers, MPI, or copies), as the reference's own NCCL wrapper does.  One
 * handle per rank holds the rank's block of the x-y decomposition with a
 * one-cell ring; hicarw_dist_configure marks the ring sides that border another
 * rank (bits 1 west, 2 east, 4 south, 8 north): their cells are halo cells,
 * filled by the caller, excluded from the reductions, and zero inside the
 * preconditioner (block Jacobi, or a block V-cycle, as :1262-1266).  The
 * operator comes from hicarw_set_coefs (probed) or calibration; FP64 Krylov
 * vectors, the reference schedule.  One iteration, with tot the caller's
 * buffers and "allreduce" the sum over ranks:
 *   hicarw_dist_setup(rhs) -> allreduce(tot[3]) -> hicarw_dist_apply(0, tot)   (once)
 *   hicarw_dist_precond(0); exchange faces of p^ (hicarw_dist_face vec 0)
 *   hicarw_dist_spmv(0) -> allreduce(tot[1]) -> hicarw_dist_apply(1, tot)
 *   hicarw_dist_precond(1); exchange faces of s^ (vec 1)
 *   hicarw_dist_spmv(1) -> allreduce(tot[5]) -> hicarw_dist_apply(2, tot)
 *   hicarw_dist_update(); hicarw_dist_state(&stop) -- until stop.
 * A face is (nz+2)(ny+2) FP64 values (west/east, side 0/1) or (nx+2)(nz+2)
 * (south/north, 2/3): pack the owned face next to a side (unpack = 0) into the
 * buffer sent to that neighbour, unpack (1) what it sent into that side's halo.
 * tot pointers follow mem_kind; the solution is read with hicarw_get_lambda. */
int hicarw_dist_configure(hicarw_handle *h, int edges);
int hicarw_dist_setup(hicarw_handle *h, const double *rhs, double *tot3, int mem_kind, void *stream);
int hicarw_dist_apply(hicarw_handle *h, int kind, const double *tot, int mem_kind, void *stream);
int hicarw_dist_precond(hicarw_handle *h, int which, void *stream);
int hicarw_dist_face(hicarw_handle *h, int vec, int side, double *buf, int unpack, void *stream);
int hicarw_dist_spmv(hicarw_handle *h, int which, double *tot, int mem_kind, void *stream);
int hicarw_dist_update(hicarw_handle *h, void *stream);
int hicarw_dist_state(hicarw_handle *h, int *stop, hicarw_stats *stats, void *stream);

/* Kernel tuning of one handle (no counterpart in the reference; the batched
 * solver's autotuner sets it per subdomain size): spmv_levels = levels per work
 * item of the float4 column-marching operator kernels (the z-march depth; 0 =
 * the default 16), mg_post_feed = 1 tensor-copy-fed / 0 register-fed multigrid
 * post-smoother on the wide levels (-1 = the default choice).  Results do not
 * depend on either. */
int hicarw_set_kernel_tuning(hicarw_handle *h, int spmv_levels, int mg_post_feed);

/* Test hook of the bounded device-side waits (no counterpart in the reference):
 * one kernel waits, through the same bounded mbarrier wait as the tensor-copy
 * smoother and the tensor-core convolutions, on a barrier that nothing completes,
 * with a limit of limit_us (1 .. 100000) microseconds.  It gives up, records the
 * error flag and returns, with nothing in flight; this call then returns
 * HICARW_ERR_TIMEOUT as a timed-out solve does, and clears the flag, so that
 * the handle and the GPU stay usable. */
int hicarw_debug_wait_timeout(hicarw_handle *h, double limit_us, void *stream);

/* Last error string of this handle (valid until its next call); h = NULL: the
 * last error of this thread's calls that take no handle (the batch entry points,
 * a failed hicarw_init_iter_winds). */
const char *hicarw_last_error(hicarw_handle *h);

/* ---- batched solves of independent, unevenly sized subdomains (no reference counterpart) ----
 * A batch borrows n calibrated handles (probed operator, HICARW_SOLVER_REFERENCE,
 * FP64 Krylov; Jacobi or multigrid preconditioner) and solves all of them in one
 * CUDA graph launch: per subdomain the set-up and a device-driven WHILE loop of
 * BiCGStab iterations, the subdomains spread over `lanes` concurrent chains.
 * Stalled multigrid solves fall back to the reference solve (status 3) as in
 * hicarw_calc_iter_winds.  All item pointers are device pointers in the layouts
 * of hicarw_calc_iter_winds; a handle may belong to one batch at a time. */
typedef struct hicarw_batch_item {
    const float *alpha, *div, *density; /* density may be NULL when adv_den == 0 */
    float *u, *v, *w;
} hicarw_batch_item;
int hicarw_batch_create(int n, hicarw_handle *const *handles, hicarw_batch **out);
int hicarw_batch_destroy(hicarw_batch *b);
/* lanes <= 0: one chain per subdomain; chunk: BiCGStab iterations per loop body (1..64). */
int hicarw_batch_config(hicarw_batch *b, int lanes, int chunk);
int hicarw_batch_get_config(const hicarw_batch *b, int *lanes, int *chunk);
/* Solve every subdomain (cold != 0 starts from lambda = 0, else from the last
 * solution, as calc_iter_winds) and correct its winds; stats: n entries (or NULL). */
int hicarw_batch_calc_iter_winds(hicarw_batch *b, const hicarw_batch_item *items, int adv_den, int cold, void *stream,
                                 hicarw_stats *stats);
/* Per-subdomain latency of the last batched call (n entries): ms from the start of
 * the batch graph to the end of that subdomain's solve loop (%globaltimer). */
int hicarw_batch_latencies(hicarw_batch *b, double *ms);
/* Time cold solves (winds untouched) for lanes in {1, 4, 16, 64} (at most n) and
 * chunk in {4, 8}, keep the fastest configuration; *best_ms its batch time. */
int hicarw_batch_autotune(hicarw_batch *b, const hicarw_batch_item *items, int adv_den, void *stream, double *best_ms);

/* Number of kernels this library has launched since load (graph nodes included). */
long long hicarw_kernel_launches(void);
/* Multigrid post-smoother launches enqueued through the tensor-copy (TMA) kernel
 * since load (a launch captured into a CUDA graph counts once).  Wide levels use
 * it unless the environment sets HICARW_MG_TMA=0 as the V-cycle is built (then
 * the register-fed kernel runs; both give bit-identical results). */
long long hicarw_mg_tma_launches(void);

/* ---- the steps either side of the solve in update_winds (wind.F90) ----
 * Device pointers only (mem_kind must be HICARW_MEM_DEVICE); caller layouts as
 * hicarw_calc_iter_winds: cells (nx, nz, ny), u (nx+1, nz, ny), v (nx, nz, ny+1).
 * Stream-ordered, FP32 in Fortran's order of operations. */
/* calc_w_real (wind.F90:1175-1227): w_real = u dz/dx + v dz/dy (face means) + the
 * mean of w_grid * jacobian_w over the cell's two w levels; w_grid may be NULL (zero). */
int hicarw_calc_w_real(hicarw_handle *h, const float *u, const float *v, const float *w_grid, float *w_real,
                       int mem_kind, void *stream);
/* calc_idealized_wgrid (wind.F90:940-998): the w_grid predictor w = stagger(w_real -
 * calc_w_real(u, v, 0)) / jacobian_w, zero on the top level (u, v: the dqdt winds). */
int hicarw_calc_idealized_wgrid(hicarw_handle *h, const float *u, const float *v, const float *w_real, float *w,
                                int mem_kind, void *stream);
/* balance_uvw + calc_w (wind.F90:123-248): w from the horizontal divergence of u, v
 * (use_dqdt selects the divergence form of the dqdt winds, as calc_divergence). */
int hicarw_balance_uvw(hicarw_handle *h, const float *u, const float *v, const float *density, float *w, int adv_den,
                       int use_dqdt, int mem_kind, void *stream);
/* update_stability (wind.F90:1421-1565): the bulk Richardson number blk_ri of each
 * column (its stability between the surface and the level ~100 m above it, and
 * the shear of the mean wind at level 5 over that depth) and, when froude_mode !=
 * 0 (alpha_const < 0 with iterative winds), the Froude number of every cell: the
 * mean wind speed over the local stability (surface potential temperature as the
 * reference) times the blocking height of the cell's wind-direction sector,
 * froude_terrain (nx, nz, ny, nsect) with 5-degree sectors (nsect = 72 in HICAR;
 * domain%vars_4d froude_terrain).  froude is 0.1 and blk_ri 10 on the top level,
 * froude 0.1 everywhere when froude_mode == 0.  u, v are the dqdt winds, z the
 * mass-level heights, theta the potential temperature (nx, nz, ny); nz >= 5. */
int hicarw_update_stability(hicarw_handle *h, const float *u, const float *v, const float *z, const float *theta,
                            const float *froude_terrain, int nsect, int froude_mode, float *froude, float *blk_ri,
                            int mem_kind, void *stream);
/* calc_alpha (wind.F90:1102-1173): alpha(Froude) in [0.2, 2], 0.2 on the top level,
 * the `halo` outermost rows / columns copied from the first tile row / column. */
int hicarw_calc_alpha(hicarw_handle *h, const float *froude, float *alpha, int halo, int mem_kind, void *stream);
/* smooth_array of alpha (update_winds :784, array_utilities.F90:322-397, ydim 3):
 * nsmooths passes of the (2 window + 1)^2 x-y box mean with clamped edges. */
int hicarw_smooth_alpha(hicarw_handle *h, float *alpha, int window, int nsmooths, int mem_kind, void *stream);

/* ---- learned preconditioner: tensor-core convolutions (no reference counterpart) ----
 * Activation tensors use the "act layout": BF16, channels in groups of 8,
 * element (c, i, k, j) of an (nx, nz, ny) grid at 16-byte unit
 * (((j+1)*(nz+2) + (k+1))*(C/8) + c/8)*PX + (i+1), lane c%8, with
 * PX = hicarw_nn_act_pitch(nx); halo cells are zero.  Weights are FP32
 * [27][cin][cout] with tap t = (dj+1)*9 + (dk+1)*3 + (di+1).  Supported
 * (cin, cout): (16,16), (16,32), (32,32), (32,16).  All pointers are device
 * pointers; the calls are synchronous on `stream`. */
int hicarw_nn_act_pitch(int nx);
/* out = epilogue(bias + conv3x3x3(in)); epilogue: + skip, ReLU (relu != 0),
 * zero where mask <= 0.  transpose != 0 runs the data-gradient convolution
 * (cout -> cin channels, flipped taps).  out0 (optional) receives channel 0 in
 * FP32 at the interior index (j*nz + k)*nx + i. */
int hicarw_nn_conv3(int cin, int cout, int nx, int ny, int nz, const void *in, const float *w, const float *bias,
                    const void *skip, const void *mask, int relu, int transpose, void *out, float *out0, void *stream);
/* Mean duration in ms (CUDA events) of `reps` forward launches (bias + ReLU), weights packed once. */
int hicarw_nn_conv3_time(int cin, int cout, int nx, int ny, int nz, const void *in, const float *w, const float *bias,
                         void *out, int reps, void *stream, float *ms);
/* dw[t][ci][co] += sum_v dy[v][co] x[v + off(t)][ci];  db[co] += sum_v dy[v][co]. */
int hicarw_nn_conv3_wgrad(int cin, int cout, int nx, int ny, int nz, const void *x, const void *dy, float *dw,
                          float *db, void *stream);

/* ---- learned preconditioner: the U-Net (no reference counterpart) ----
 * A 3-level U-Net of the convolutions above (levels: full grid, x-y halved,
 * x-y quartered; 16/32/32 channels; ReLU; 2x2 average pooling; nearest
 * upsampling; additive skips) maps the features of a residual r (r / rms(r)
 * and the 14 stencil ratios coef_q / coef_A) to z = O_0 rms(r) / coef_A, a
 * correction of the Jacobi step it starts from.  Parameters are FP32 (the
 * 7 convolutions' [27][cin][cout] weights, each followed by its bias, in order
 * a..g); activations BF16.  A network object owns the activations of one grid
 * size; copy parameters between objects with get/set_params. */
int hicarw_unet_create(int nx, int ny, int nz, unsigned long long seed, hicarw_unet **out);
int hicarw_unet_destroy(hicarw_unet *n);
int hicarw_unet_grid(const hicarw_unet *n, int *nx, int *ny, int *nz);
long long hicarw_unet_num_params(const hicarw_unet *n);
int hicarw_unet_get_params(hicarw_unet *n, float *out, int mem_kind, void *stream);
int hicarw_unet_set_params(hicarw_unet *n, const float *in, int mem_kind, void *stream);
int hicarw_unet_get_grads(hicarw_unet *n, float *out, int mem_kind, void *stream);
int hicarw_unet_zero_grads(hicarw_unet *n, void *stream);
/* Input features of r (device FP64, (nx+2, nz+2, ny+2)) for the handle's probed
 * operator into x0 (device, act layout, 16 channels); rms(r) to *rms (host). */
int hicarw_unet_features(hicarw_unet *n, hicarw_handle *h, const double *r, void *x0, float *rms, void *stream);
/* Forward pass from features x0; out0 (device, optional) receives O_0 at (j*nz + k)*nx + i. */
int hicarw_unet_forward(hicarw_unet *n, const void *x0, float *out0, void *stream);
/* After a forward pass: loss = weight * mean((O_0 - target)^2) (to *loss, host),
 * and the parameter gradients of that loss added to the accumulated gradients. */
int hicarw_unet_backward(hicarw_unet *n, const float *target, float weight, float *loss, void *stream);
/* After a forward pass on the features of a unit-rms residual rhat (device FP32
 * (ny, nz, nx)): loss = weight * mean((A z - rhat)^2) with z = O_0 / coef_A and A
 * the operator of the (15, ny, nz, nx) FP32 coefficients coef (hicarw_get_coefs
 * layout, zero values outside the interior); gradients accumulated as above. */
int hicarw_unet_backward_residual(hicarw_unet *n, const float *coef, const float *rhat, float weight, float *loss,
                                  void *stream);
/* Adam step (beta 0.9 / 0.999) with the mean of the accumulated gradients; clears them. */
int hicarw_unet_adam_step(hicarw_unet *n, float lr, void *stream);
/* z = M(r) on device FP64 (nx+2, nz+2, ny+2) vectors (ghost cells of z untouched). */
int hicarw_unet_apply(hicarw_unet *n, hicarw_handle *h, const double *r, double *z, void *stream);
/* Attach the network used by HICARW_PRECOND_LEARNED (same grid; NULL detaches). */
int hicarw_set_learned_precond(hicarw_handle *h, hicarw_unet *n);

#ifdef __cplusplus
}
#endif
#endif /* HICARW_H */
