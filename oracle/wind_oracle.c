/*
 * wind_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of HICAR's iterative mass-conserving wind solver
 * (module wind_iterative, src/physics/wind_iterative.F90) and of the two
 * wind.F90 routines that define its operator and right-hand side
 * (calc_divergence, calibrate_projection_operator).  Only tests/, the smoke
 * entry and the CPU-baseline leg of bench.py may load this library.
 *
 * Parity status: UNPINNED by golden vectors.  The reference ships no golden
 * vector or known-answer test for this path (its only unit test asserts that
 * max|div| decreases, tests/unit/test_wind_iterative.F90:139-152) and it cannot
 * be compiled in this environment (Fortran 2008 + MPI + NetCDF + OpenACC).
 * The restatement follows the reference statement by statement; every
 * function cites the lines it restates.  Known-answer tests in tests/ pin it
 * (manufactured solutions, probe == analytic composition, the reference unit
 * test's divergence-reduction assertion).
 *
 * Precision.  Built twice from this one file:
 *   - reference precision (default): fields, metrics, coefficients, the
 *     divergence and the lambda->wind correction in FP32 ("real"), Krylov
 *     vectors and reductions in FP64 ("real(c_double)"), exactly as the
 *     reference declares them (wind_iterative.F90:86-92,110-122);
 *   - ORC_FLD_DOUBLE: every field in FP64 (the "FP64 oracle").
 * Floating-point statements keep Fortran's left-to-right evaluation order;
 * the recipe compiles with -ffp-contract=off so no multiply-add is fused.
 *
 * Index conventions at one rank (wind_iterative.F90:2279-2302, grid_obj.F90:186-204):
 *   cell arrays       (1:nx, 1:nz, 1:ny)        i fastest, then k, then j
 *   u-staggered       (1:nx+1, 1:nz, 1:ny)
 *   v-staggered       (1:nx, 1:nz, 1:ny+1)
 *   dz_if             (1:nx, 1:nz+1, 1:ny)
 *   Krylov vectors    (0:nx+1, 0:nz+1, 0:ny+1)  rows: mx=nx+2, mz=nz+2, my=ny+2
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_FLD_DOUBLE
typedef double fld;
#define FLD_SQRT sqrt
#else
typedef float fld;
#define FLD_SQRT sqrtf /* single-precision square root, as Fortran's sqrt of a real */
#endif

#define NCOEF 15
enum { CA = 0, CB, CC, CD, CE, CF, CG, CH, CI, CJ, CK, CL, CM, CN, CO };

typedef struct orc_domain {
    int nx, ny, nz;
    fld dx;
    const fld *jacobian, *jacobian_u, *jacobian_v, *jacobian_w; /* cell, u, v, cell */
    const fld *dzdx, *dzdy, *dzdx_u, *dzdy_v;                   /* cell, cell, u, v */
    const fld *advection_dz;                                    /* cell */
    const fld *neighbor_terrain;                                /* (nx, ny) */
    const fld *density;                                         /* cell */
    const fld *mapfac_mx_u, *mapfac_my_v;                       /* (nx+1,ny), (nx,ny+1) */
    const fld *mapfac_my_u, *mapfac_mx_v, *mapfac_mxy;          /* (nx+1,ny), (nx,ny+1), (nx,ny) */
} orc_domain;

typedef struct orc_stats {
    int status, iters, sweeps, retries, fatal;
    double res0, res_final, b_norm, target;
} orc_stats;

typedef struct orc_solver {
    orc_domain d;
    int nx, ny, nz, mx, my, mz;
    size_t nrows, ncell;
    fld dx;
    /* module copies (wind_iterative.F90:86-92) */
    fld *dz_if, *dzdx_surf, *dzdy_surf, *adv_dz_col, *alpha, *div;
    fld *coef[NCOEF];
    /* Krylov state (wind_iterative.F90:110-122) */
    double *x, *r, *rhat, *p, *phat, *v, *s, *shat, *t, *rhs, *Dinv, *pres;
    int structure_uploaded, operator_probed, precond_n_sweeps, max_iters;
    double tol_rel, tol_abs;
    double *hist;   /* recurrence residual norm per iteration of the last bicgstab_solve */
    int hist_len, hist_cap;
    orc_stats last;
} orc_solver;

static const double breakdown_eps = 1.0e-30; /* wind_iterative.F90:61 */
#define BASE_PREC_SWEEPS 2                   /* wind_iterative.F90:75 */
#define MAX_PREC_SWEEPS 4                    /* wind_iterative.F90:76 */

/* ---- index helpers (1-based Fortran indices) ---- */
#define IC(s, i, k, j) ((size_t)((i) - 1) + (size_t)(s)->nx * ((size_t)((k) - 1) + (size_t)(s)->nz * (size_t)((j) - 1)))
#define IU(s, i, k, j) ((size_t)((i) - 1) + (size_t)((s)->nx + 1) * ((size_t)((k) - 1) + (size_t)(s)->nz * (size_t)((j) - 1)))
#define IV(s, i, k, j) IC(s, i, k, j)
#define IZ(s, i, k, j) ((size_t)((i) - 1) + (size_t)(s)->nx * ((size_t)((k) - 1) + (size_t)((s)->nz + 1) * (size_t)((j) - 1)))
#define I2(s, i, j) ((size_t)((i) - 1) + (size_t)(s)->nx * (size_t)((j) - 1))
#define I2U(s, i, j) ((size_t)((i) - 1) + (size_t)((s)->nx + 1) * (size_t)((j) - 1))
#define IK(s, i, k, j) ((size_t)(i) + (size_t)(s)->mx * ((size_t)(k) + (size_t)(s)->mz * (size_t)(j)))

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_fld_bytes(void) { return (int)sizeof(fld); }

/* ------------------------------------------------------------------------ */
/* init_module_vars: wind_iterative.F90:2274-2421 (one rank: i_s=1, i_e=nx). */
/* ------------------------------------------------------------------------ */
static void init_module_vars(orc_solver *s)
{
    const orc_domain *d = &s->d;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    fld dx = s->dx;
    /* dz_if(i,k,j) = (adz(k) + adz(k-1)) / 2 for k=k_s+1..k_e   (:2339-2345) */
#pragma omp parallel for
    for (int j = 1; j <= ny; j++) {
        for (int k = 2; k <= nz; k++)
            for (int i = 1; i <= nx; i++)
                s->dz_if[IZ(s, i, k, j)] = (d->advection_dz[IC(s, i, k, j)] + d->advection_dz[IC(s, i, k - 1, j)]) / (fld)2;
        /* (:2346-2354) */
        for (int i = 1; i <= nx; i++) {
            s->dz_if[IZ(s, i, 1, j)] = d->advection_dz[IC(s, i, 1, j)];
            s->dz_if[IZ(s, i, nz + 1, j)] = d->advection_dz[IC(s, i, nz, j)];
            s->dzdx_surf[I2(s, i, j)] = d->dzdx[IC(s, i, 1, j)];
            s->dzdy_surf[I2(s, i, j)] = d->dzdy[IC(s, i, 1, j)];
        }
    }
    /* centred terrain slope on interior columns (:2382-2393); i_s_bnd = 2, i_e_bnd = nx-1 */
#pragma omp parallel for
    for (int j = 1; j <= ny; j++)
        for (int i = 2; i <= nx - 1; i++)
            s->dzdx_surf[I2(s, i, j)] = (d->neighbor_terrain[I2(s, i + 1, j)] - d->neighbor_terrain[I2(s, i - 1, j)]) / (2 * dx);
#pragma omp parallel for
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 1; i <= nx; i++)
            s->dzdy_surf[I2(s, i, j)] = (d->neighbor_terrain[I2(s, i, j + 1)] - d->neighbor_terrain[I2(s, i, j - 1)]) / (2 * dx);
    /* adv_dz_col(k) = adv_dz(i_s, k, j_s)  (:2394-2397) */
    for (int k = 1; k <= nz; k++) s->adv_dz_col[k - 1] = d->advection_dz[IC(s, 1, k, 1)];
}

/* ------------------------------------------------------------------------ */
/* initialize_coefs + update_coefs_host: wind_iterative.F90:2424-2552.      */
/* ------------------------------------------------------------------------ */
static void update_coefs_host(orc_solver *s)
{
    const orc_domain *d = &s->d;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    fld dx = s->dx;
    const fld *adz = d->advection_dz; /* only column (i_s, :, j_s) is read, as in the reference */
#define ADZ(k) adz[IC(s, 1, (k), 1)]
#pragma omp parallel for
    for (int j = 1; j <= ny; j++) {
        for (int k = 1; k <= nz; k++) {
            for (int i = 1; i <= nx; i++) {
                size_t c = IC(s, i, k, j);
                fld dzdx_k = d->dzdx[c], dzdy_k = d->dzdy[c], a_k = s->alpha[c];
                fld M_up, M_dwn;
                if (k == 1) { /* (:2494-2505) */
                    fld dzdx_p = d->dzdx[IC(s, i, k + 1, j)], dzdy_p = d->dzdy[IC(s, i, k + 1, j)], a_p = s->alpha[IC(s, i, k + 1, j)];
                    fld jw = d->jacobian_w[c];
                    M_up = dzdx_k * (dzdx_k * ADZ(k + 1) + dzdx_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
                    M_dwn = dzdx_k * s->dzdx_surf[I2(s, i, j)];
                    M_up = M_up + dzdy_k * (dzdy_k * ADZ(k + 1) + dzdy_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
                    M_dwn = M_dwn + dzdy_k * s->dzdy_surf[I2(s, i, j)];
                    M_up = M_up + (a_k * a_k * ADZ(k + 1) + a_p * a_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
                    M_dwn = M_dwn + a_k * a_k;
                } else if (k == nz) { /* (:2506-2524) */
                    fld dzdx_m = d->dzdx[IC(s, i, k - 1, j)], dzdy_m = d->dzdy[IC(s, i, k - 1, j)], a_m = s->alpha[IC(s, i, k - 1, j)];
                    fld jwm = d->jacobian_w[IC(s, i, k - 1, j)];
                    M_up = dzdx_k * (dzdx_k * ADZ(k) + dzdx_k * ADZ(k)) / (ADZ(k) + ADZ(k));
                    M_dwn = dzdx_k * (dzdx_k * ADZ(k - 1) + dzdx_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
                    M_up = M_up + dzdy_k * (dzdy_k * ADZ(k) + dzdy_k * ADZ(k)) / (ADZ(k) + ADZ(k));
                    M_dwn = M_dwn + dzdy_k * (dzdy_k * ADZ(k - 1) + dzdy_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
                    M_up = M_up + (a_k * a_k * ADZ(k) + a_k * a_k * ADZ(k)) / (ADZ(k) + ADZ(k));
                    M_dwn = M_dwn + (a_k * a_k * ADZ(k - 1) + a_m * a_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
                } else { /* (:2525-2543) */
                    fld dzdx_p = d->dzdx[IC(s, i, k + 1, j)], dzdy_p = d->dzdy[IC(s, i, k + 1, j)], a_p = s->alpha[IC(s, i, k + 1, j)];
                    fld dzdx_m = d->dzdx[IC(s, i, k - 1, j)], dzdy_m = d->dzdy[IC(s, i, k - 1, j)], a_m = s->alpha[IC(s, i, k - 1, j)];
                    fld jw = d->jacobian_w[c], jwm = d->jacobian_w[IC(s, i, k - 1, j)];
                    M_up = dzdx_k * (dzdx_k * ADZ(k + 1) + dzdx_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
                    M_dwn = dzdx_k * (dzdx_k * ADZ(k - 1) + dzdx_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
                    M_up = M_up + dzdy_k * (dzdy_k * ADZ(k + 1) + dzdy_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
                    M_dwn = M_dwn + dzdy_k * (dzdy_k * ADZ(k - 1) + dzdy_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
                    M_up = M_up + (a_k * a_k * ADZ(k + 1) + a_p * a_p * ADZ(k)) / (ADZ(k) + ADZ(k + 1)) / jw;
                    M_dwn = M_dwn + (a_k * a_k * ADZ(k - 1) + a_m * a_m * ADZ(k)) / (ADZ(k) + ADZ(k - 1)) / jwm;
                }
                /* (:2545-2546) */
                fld Bv = M_up / (d->jacobian[c] * ADZ(k) * s->dz_if[IZ(s, 1, k + 1, 1)]);
                fld Cv = M_dwn / (d->jacobian[c] * ADZ(k) * s->dz_if[IZ(s, 1, k, 1)]);
                /* A = -4/dx^2 - B - C before the cross term (:2549) */
                fld Av = (fld)-4 / (dx * dx) - Bv - Cv;
                /* X cross term (:2551-2553) */
                fld mixed_denom = (s->dz_if[IZ(s, i, k + 1, j)] + s->dz_if[IZ(s, i, k, j)]) * 2 * dx;
                fld X = -((d->dzdx_u[IU(s, i + 1, k, j)] / d->jacobian_u[IU(s, i + 1, k, j)] - d->dzdx_u[IU(s, i, k, j)] / d->jacobian_u[IU(s, i, k, j)]) +
                          (d->dzdy_v[IV(s, i, k, j + 1)] / d->jacobian_v[IV(s, i, k, j + 1)] - d->dzdy_v[IV(s, i, k, j)] / d->jacobian_v[IV(s, i, k, j)])) /
                        mixed_denom;
                s->coef[CA][c] = Av;
                s->coef[CB][c] = Bv + X;
                s->coef[CC][c] = Cv - X;
            }
        }
    }
#undef ADZ
}

static void initialize_coefs(orc_solver *s)
{
    const orc_domain *d = &s->d;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    fld dx = s->dx;
    fld inv = (fld)1.0 / (dx * dx); /* D=E=F=G = 1/dx^2 (:2448-2451) */
#pragma omp parallel for
    for (int j = 1; j <= ny; j++)
        for (int k = 1; k <= nz; k++) {
            /* mixed_denom = 2*dx*(dz_if(i_s,k+1,j_s) + dz_if(i_s,k,j_s)) (:2454) */
            fld mixed_denom = 2 * dx * (s->dz_if[IZ(s, 1, k + 1, 1)] + s->dz_if[IZ(s, 1, k, 1)]);
            for (int i = 1; i <= nx; i++) {
                size_t c = IC(s, i, k, j);
                fld gx = d->dzdx[c] / d->jacobian[c], gy = d->dzdy[c] / d->jacobian[c];
                fld ux1 = d->dzdx_u[IU(s, i + 1, k, j)] / d->jacobian_u[IU(s, i + 1, k, j)];
                fld ux0 = d->dzdx_u[IU(s, i, k, j)] / d->jacobian_u[IU(s, i, k, j)];
                fld vy1 = d->dzdy_v[IV(s, i, k, j + 1)] / d->jacobian_v[IV(s, i, k, j + 1)];
                fld vy0 = d->dzdy_v[IV(s, i, k, j)] / d->jacobian_v[IV(s, i, k, j)];
                s->coef[CA][c] = 1;
                s->coef[CB][c] = 0;
                s->coef[CC][c] = 0;
                s->coef[CD][c] = inv;
                s->coef[CE][c] = inv;
                s->coef[CF][c] = inv;
                s->coef[CG][c] = inv;
                /* (:2455-2462) */
                s->coef[CH][c] = -(gx + ux1) / mixed_denom;
                s->coef[CI][c] = (gx + ux0) / mixed_denom;
                s->coef[CL][c] = -(gy + vy1) / mixed_denom;
                s->coef[CM][c] = (gy + vy0) / mixed_denom;
                s->coef[CJ][c] = (gx + ux1) / mixed_denom;
                s->coef[CK][c] = -(gx + ux0) / mixed_denom;
                s->coef[CN][c] = (gy + vy1) / mixed_denom;
                s->coef[CO][c] = -(gy + vy0) / mixed_denom;
            }
        }
    update_coefs_host(s);
}

/* update_coefs_gpu: wind_iterative.F90:2555-2603 (alpha refresh, analytic operator only). */
static void update_coefs_gpu(orc_solver *s)
{
    const orc_domain *d = &s->d;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    fld dx = s->dx;
#pragma omp parallel for
    for (int j = 1; j <= ny; j++)
        for (int k = 1; k <= nz; k++)
            for (int i = 1; i <= nx; i++) {
                size_t c = IC(s, i, k, j);
                fld adz_k = s->adv_dz_col[k - 1];
                fld dzdx_k = d->dzdx[c], dzdy_k = d->dzdy[c], a_k = s->alpha[c];
                fld M_up, M_dwn;
                if (k == nz) {
                    M_up = dzdx_k * dzdx_k + dzdy_k * dzdy_k + a_k * a_k;
                } else {
                    fld adz_p = s->adv_dz_col[k], sum_up = adz_k + adz_p;
                    size_t cp = IC(s, i, k + 1, j);
                    fld jw = d->jacobian_w[c];
                    M_up = dzdx_k * (dzdx_k * adz_p + d->dzdx[cp] * adz_k) / sum_up / jw +
                           dzdy_k * (dzdy_k * adz_p + d->dzdy[cp] * adz_k) / sum_up / jw +
                           (a_k * a_k * adz_p + s->alpha[cp] * s->alpha[cp] * adz_k) / sum_up / jw;
                }
                if (k == 1) {
                    M_dwn = dzdx_k * s->dzdx_surf[I2(s, i, j)] + dzdy_k * s->dzdy_surf[I2(s, i, j)] + a_k * a_k;
                } else {
                    fld adz_m = s->adv_dz_col[k - 2], sum_dw = adz_k + adz_m;
                    size_t cm = IC(s, i, k - 1, j);
                    fld jwm = d->jacobian_w[cm];
                    M_dwn = dzdx_k * (dzdx_k * adz_m + d->dzdx[cm] * adz_k) / sum_dw / jwm +
                            dzdy_k * (dzdy_k * adz_m + d->dzdy[cm] * adz_k) / sum_dw / jwm +
                            (a_k * a_k * adz_m + s->alpha[cm] * s->alpha[cm] * adz_k) / sum_dw / jwm;
                }
                fld Bv = M_up / (d->jacobian[c] * adz_k * s->dz_if[IZ(s, 1, k + 1, 1)]);
                fld Cv = M_dwn / (d->jacobian[c] * adz_k * s->dz_if[IZ(s, 1, k, 1)]);
                fld mixed = (s->dz_if[IZ(s, i, k + 1, j)] + s->dz_if[IZ(s, i, k, j)]) * (fld)2.0 * dx;
                fld X = -((d->dzdx_u[IU(s, i + 1, k, j)] / d->jacobian_u[IU(s, i + 1, k, j)] - d->dzdx_u[IU(s, i, k, j)] / d->jacobian_u[IU(s, i, k, j)]) +
                          (d->dzdy_v[IV(s, i, k, j + 1)] / d->jacobian_v[IV(s, i, k, j + 1)] - d->dzdy_v[IV(s, i, k, j)] / d->jacobian_v[IV(s, i, k, j)])) /
                        mixed;
                Bv = Bv + X;
                Cv = Cv - X;
                s->coef[CB][c] = Bv;
                s->coef[CC][c] = Cv;
                s->coef[CA][c] = (fld)-4.0 / (dx * dx) - Bv - Cv;
            }
}

/* ------------------------------------------------------------------------ */
/* spmv: wind_iterative.F90:813-1027                                        */
/* ------------------------------------------------------------------------ */
void orc_spmv(orc_solver *s, const double *x, double *y)
{
    int nx = s->nx, ny = s->ny, nz = s->nz, mx = s->mx, my = s->my, mz = s->mz;
    double dx = (double)s->dx;
    double two_dx = 2.0 * dx, inv_dx2 = 1.0 / (dx * dx), neg_4_inv_dx2 = -4.0 * inv_dx2;
    (void)nx; (void)ny; (void)nz;
    /* lateral identity rows (:839-871 / :916-948) */
#pragma omp parallel for
    for (int j = 0; j < my; j++)
        for (int k = 0; k < mz; k++) {
            y[IK(s, 0, k, j)] = x[IK(s, 0, k, j)];
            y[IK(s, mx - 1, k, j)] = x[IK(s, mx - 1, k, j)];
        }
#pragma omp parallel for
    for (int k = 0; k < mz; k++)
        for (int i = 0; i < mx; i++) {
            y[IK(s, i, k, 0)] = x[IK(s, i, k, 0)];
            y[IK(s, i, k, my - 1)] = x[IK(s, i, k, my - 1)];
        }
    if (s->operator_probed) {
#pragma omp parallel for
        for (int j = 1; j <= my - 2; j++) {
            /* ghost-plane identity rows (:873-881) */
            for (int i = 1; i <= mx - 2; i++) {
                y[IK(s, i, 0, j)] = x[IK(s, i, 0, j)];
                y[IK(s, i, mz - 1, j)] = x[IK(s, i, mz - 1, j)];
            }
            /* probed 15-point interior (:883-907) */
            for (int k = 1; k <= mz - 2; k++)
                for (int i = 1; i <= mx - 2; i++) {
                    size_t c = IC(s, i, k, j);
#define CF64(n) ((double)s->coef[n][c])
                    y[IK(s, i, k, j)] = CF64(CO) * x[IK(s, i, k - 1, j - 1)] + CF64(CG) * x[IK(s, i, k, j - 1)] +
                                        CF64(CM) * x[IK(s, i, k + 1, j - 1)] + CF64(CK) * x[IK(s, i - 1, k - 1, j)] +
                                        CF64(CC) * x[IK(s, i, k - 1, j)] + CF64(CJ) * x[IK(s, i + 1, k - 1, j)] +
                                        CF64(CE) * x[IK(s, i - 1, k, j)] + CF64(CA) * x[IK(s, i, k, j)] +
                                        CF64(CD) * x[IK(s, i + 1, k, j)] + CF64(CI) * x[IK(s, i - 1, k + 1, j)] +
                                        CF64(CB) * x[IK(s, i, k + 1, j)] + CF64(CH) * x[IK(s, i + 1, k + 1, j)] +
                                        CF64(CN) * x[IK(s, i, k - 1, j + 1)] + CF64(CF) * x[IK(s, i, k, j + 1)] +
                                        CF64(CL) * x[IK(s, i, k + 1, j + 1)];
                }
        }
        return;
    }
#pragma omp parallel for
    for (int j = 1; j <= my - 2; j++) {
        for (int i = 1; i <= mx - 2; i++) {
            /* top BC k=mz-1 (:950-960) */
            y[IK(s, i, mz - 1, j)] = (x[IK(s, i, mz - 1, j)] - x[IK(s, i, mz - 2, j)]) / (double)s->dz_if[IZ(s, i, mz - 1, j)];
            /* bottom 10-point terrain BC k=0 (:962-988) */
            double dzdx_s = (double)s->dzdx_surf[I2(s, i, j)];
            double dzdy_s = (double)s->dzdy_surf[I2(s, i, j)];
            double dz_kp1 = (double)s->dz_if[IZ(s, i, 1, j)];
            double al = (double)s->alpha[IC(s, i, 1, j)];
            double denom = 2.0 * (dzdx_s * dzdx_s + dzdy_s * dzdy_s + al * al) / (double)s->d.jacobian[IC(s, i, 1, j)];
            y[IK(s, i, 0, j)] = (dzdy_s / (denom * two_dx)) * x[IK(s, i, 0, j - 1)] + (dzdy_s / (denom * two_dx)) * x[IK(s, i, 1, j - 1)] +
                                (dzdx_s / (denom * two_dx)) * x[IK(s, i - 1, 0, j)] + (-1.0 / dz_kp1) * x[IK(s, i, 0, j)] +
                                (-dzdx_s / (denom * two_dx)) * x[IK(s, i + 1, 0, j)] + (dzdx_s / (denom * two_dx)) * x[IK(s, i - 1, 1, j)] +
                                (1.0 / dz_kp1) * x[IK(s, i, 1, j)] + (-dzdx_s / (denom * two_dx)) * x[IK(s, i + 1, 1, j)] +
                                (-dzdy_s / (denom * two_dx)) * x[IK(s, i, 0, j + 1)] + (-dzdy_s / (denom * two_dx)) * x[IK(s, i, 1, j + 1)];
        }
        /* analytic interior, D..G scalar, A on the fly (:990-1025) */
        for (int k = 1; k <= mz - 2; k++)
            for (int i = 1; i <= mx - 2; i++) {
                size_t c = IC(s, i, k, j);
                double b_val = CF64(CB), c_val = CF64(CC);
                double a_val = neg_4_inv_dx2 - b_val - c_val;
                y[IK(s, i, k, j)] = CF64(CO) * x[IK(s, i, k - 1, j - 1)] + inv_dx2 * x[IK(s, i, k, j - 1)] +
                                    CF64(CM) * x[IK(s, i, k + 1, j - 1)] + CF64(CK) * x[IK(s, i - 1, k - 1, j)] +
                                    c_val * x[IK(s, i, k - 1, j)] + CF64(CJ) * x[IK(s, i + 1, k - 1, j)] +
                                    inv_dx2 * x[IK(s, i - 1, k, j)] + a_val * x[IK(s, i, k, j)] +
                                    inv_dx2 * x[IK(s, i + 1, k, j)] + CF64(CI) * x[IK(s, i - 1, k + 1, j)] +
                                    b_val * x[IK(s, i, k + 1, j)] + CF64(CH) * x[IK(s, i + 1, k + 1, j)] +
                                    CF64(CN) * x[IK(s, i, k - 1, j + 1)] + inv_dx2 * x[IK(s, i, k, j + 1)] +
                                    CF64(CL) * x[IK(s, i, k + 1, j + 1)];
#undef CF64
            }
    }
}

/* extract_diagonal: wind_iterative.F90:1041-1075 */
static void extract_diagonal(orc_solver *s)
{
    int mx = s->mx, my = s->my, mz = s->mz;
#pragma omp parallel for
    for (int j = 0; j < my; j++)
        for (int k = 0; k < mz; k++)
            for (int i = 0; i < mx; i++) {
                double dd;
                if (i <= 0 || j <= 0 || i >= mx - 1 || j >= my - 1) dd = 1.0;
                else if (k >= mz - 1) dd = s->operator_probed ? 1.0 : 1.0 / (double)s->dz_if[IZ(s, i, k, j)];
                else if (k <= 0) dd = s->operator_probed ? 1.0 : -1.0 / (double)s->dz_if[IZ(s, i, k + 1, j)];
                else dd = (double)s->coef[CA][IC(s, i, k, j)];
                if (fabs(dd) < breakdown_eps) dd = copysign(breakdown_eps, dd);
                s->Dinv[IK(s, i, k, j)] = 1.0 / dd;
            }
}

/* compute_rhs_3d: wind_iterative.F90:1513-1530 */
static void compute_rhs_3d(orc_solver *s)
{
    int mx = s->mx, my = s->my, mz = s->mz;
#pragma omp parallel for
    for (int j = 0; j < my; j++)
        for (int k = 0; k < mz; k++)
            for (int i = 0; i < mx; i++) {
                if (i <= 0 || j <= 0 || i >= mx - 1 || j >= my - 1 || k <= 0 || k >= mz - 1)
                    s->rhs[IK(s, i, k, j)] = 0.0;
                else
                    s->rhs[IK(s, i, k, j)] = (double)((fld)-2.0 * s->div[IC(s, i, k, j)]);
            }
}

/* ---- vector kernels over the owned range (all rows at one rank), :1323-1506 ---- */
static void vec_zero(orc_solver *s, double *v) { memset(v, 0, s->nrows * sizeof(double)); }
static void vec_copy(orc_solver *s, double *dst, const double *src) { memcpy(dst, src, s->nrows * sizeof(double)); }
static void vec_axpby_into(orc_solver *s, double *o, double a, const double *x, double b, const double *y)
{
    ptrdiff_t n = (ptrdiff_t)s->nrows;
#pragma omp parallel for
    for (ptrdiff_t q = 0; q < n; q++) o[q] = a * x[q] + b * y[q];
}
static void vec_axpy2(orc_solver *s, double *y, double a, const double *x, double b, const double *z)
{
    ptrdiff_t n = (ptrdiff_t)s->nrows;
#pragma omp parallel for
    for (ptrdiff_t q = 0; q < n; q++) y[q] = y[q] + a * x[q] + b * z[q];
}
static void vec_p_update(orc_solver *s, double *p, const double *r, double beta, double omega, const double *v)
{
    ptrdiff_t n = (ptrdiff_t)s->nrows;
#pragma omp parallel for
    for (ptrdiff_t q = 0; q < n; q++) p[q] = r[q] + beta * (p[q] - omega * v[q]);
}
/* Deterministic reductions: one partial per j-plane, summed in plane order. */
static double vec_dot(orc_solver *s, const double *x, const double *y)
{
    size_t plane = (size_t)s->mx * s->mz;
    int my = s->my;
    double *part = (double *)malloc(sizeof(double) * my);
#pragma omp parallel for
    for (int j = 0; j < my; j++) {
        double acc = 0.0;
        const double *xa = x + plane * j, *ya = y + plane * j;
        for (size_t q = 0; q < plane; q++) acc += xa[q] * ya[q];
        part[j] = acc;
    }
    double sum = 0.0;
    for (int j = 0; j < my; j++) sum += part[j];
    free(part);
    return sum;
}
static void vec_dots_fused(orc_solver *s, const double *t, const double *sv, const double *rh, double out[5])
{
    size_t plane = (size_t)s->mx * s->mz;
    int my = s->my;
    double *part = (double *)malloc(sizeof(double) * 5 * my);
#pragma omp parallel for
    for (int j = 0; j < my; j++) {
        double ts = 0, tt = 0, rs = 0, rt = 0, ss = 0;
        for (size_t q = plane * j; q < plane * (j + 1); q++) {
            double tv = t[q], svv = sv[q], rv = rh[q];
            ts += tv * svv;
            tt += tv * tv;
            rs += rv * svv;
            rt += rv * tv;
            ss += svv * svv;
        }
        part[5 * j + 0] = ts; part[5 * j + 1] = tt; part[5 * j + 2] = rs; part[5 * j + 3] = rt; part[5 * j + 4] = ss;
    }
    for (int m = 0; m < 5; m++) out[m] = 0.0;
    for (int j = 0; j < my; j++)
        for (int m = 0; m < 5; m++) out[m] += part[5 * j + m];
    free(part);
}

/* apply_precond: wind_iterative.F90:1268-1315 (Jacobi-Richardson, zero halo) */
void orc_apply_precond(orc_solver *s, const double *in, double *out)
{
    ptrdiff_t n = (ptrdiff_t)s->nrows;
    memset(out, 0, s->nrows * sizeof(double));
#pragma omp parallel for
    for (ptrdiff_t q = 0; q < n; q++) out[q] = s->Dinv[q] * in[q];
    for (int sweep = 2; sweep <= s->precond_n_sweeps; sweep++) {
        orc_spmv(s, out, s->pres);
#pragma omp parallel for
        for (ptrdiff_t q = 0; q < n; q++) out[q] = out[q] + s->Dinv[q] * (in[q] - s->pres[q]);
    }
}

static void hist_push(orc_solver *s, double v)
{
    if (s->hist_len >= s->hist_cap) {
        s->hist_cap = s->hist_cap ? 2 * s->hist_cap : 256;
        s->hist = (double *)realloc(s->hist, sizeof(double) * s->hist_cap);
    }
    s->hist[s->hist_len++] = v;
}

/* bicgstab_solve: wind_iterative.F90:555-791 (1 rank: halo exchange / allreduce are no-ops) */
void orc_bicgstab(orc_solver *s, int max_iters, orc_stats *st)
{
    double rho, rho_new, alpha_s, beta_s, omega, sigma, ts, tt, rs, rt, ss, rnorm, rn2, target, b_norm2, red5[5];
    st->status = 1; st->iters = 0; st->res0 = 0.0; st->res_final = 0.0;
    s->hist_len = 0;
    orc_spmv(s, s->x, s->t);                              /* :589 */
    vec_axpby_into(s, s->r, 1.0, s->rhs, -1.0, s->t);     /* :590 */
    vec_copy(s, s->rhat, s->r);                           /* :592 */
    vec_copy(s, s->p, s->r);                              /* :594 */
    rho = vec_dot(s, s->rhat, s->r);                      /* :602 */
    rnorm = sqrt(vec_dot(s, s->r, s->r));                 /* :603,630 */
    b_norm2 = vec_dot(s, s->rhs, s->rhs);                 /* :604 */
    st->res0 = rnorm; st->res_final = rnorm;
    target = fmax(s->tol_abs, s->tol_rel * sqrt(b_norm2)); /* :633 */
    st->b_norm = sqrt(b_norm2); st->target = target;
    hist_push(s, rnorm);
    if (rnorm <= target) { st->status = 0; st->iters = 0; return; }
    omega = 1.0; alpha_s = 1.0;
    for (int it = 1; it <= max_iters; it++) {
        orc_apply_precond(s, s->p, s->phat);              /* :649 */
        orc_spmv(s, s->phat, s->v);                       /* :657 */
        sigma = vec_dot(s, s->rhat, s->v);                /* :662 */
        if (fabs(sigma) < breakdown_eps) { st->status = 2; st->iters = it; break; } /* :680 */
        alpha_s = rho / sigma;
        vec_axpby_into(s, s->s, 1.0, s->r, -alpha_s, s->v);   /* :690 */
        orc_apply_precond(s, s->s, s->shat);              /* :695 */
        orc_spmv(s, s->shat, s->t);                       /* :703 */
        vec_dots_fused(s, s->t, s->s, s->rhat, red5);     /* :711 */
        ts = red5[0]; tt = red5[1]; rs = red5[2]; rt = red5[3]; ss = red5[4];
        if (tt < breakdown_eps) { st->status = 2; st->iters = it; break; } /* :737 */
        omega = ts / tt;
        rho_new = rs - omega * rt;
        rn2 = ss - 2.0 * omega * ts + omega * omega * tt; /* :748 */
        if (rn2 < 0.0) rn2 = 0.0;
        rnorm = sqrt(rn2);
        st->res_final = rnorm; st->iters = it;
        hist_push(s, rnorm);
        vec_axpy2(s, s->x, alpha_s, s->phat, omega, s->shat); /* :755 */
        if (rnorm <= target) { st->status = 0; break; }
        if (fabs(omega) < breakdown_eps) { st->status = 2; break; }
        vec_axpby_into(s, s->r, 1.0, s->s, -omega, s->t);   /* :771 */
        if (fabs(rho) < breakdown_eps) { st->status = 2; break; }
        beta_s = (rho_new / rho) * (alpha_s / omega);
        vec_p_update(s, s->p, s->r, beta_s, omega, s->v);   /* :781 */
        rho = rho_new;
    }
}

/* ------------------------------------------------------------------------ */
/* calc_updated_winds: wind_iterative.F90:1742-2071 (lambda -> u, v, w_grid) */
/* u: (nx+1,nz,ny)  v: (nx,nz,ny+1)  w: (nx,nz,ny)                          */
/* ------------------------------------------------------------------------ */
void orc_calc_updated_winds(orc_solver *s, int adv_den, fld *u, fld *v, fld *w)
{
    const orc_domain *d = &s->d;
    int nx = s->nx, ny = s->ny, nz = s->nz, mx = s->mx, mz = s->mz;
    fld dx = s->dx;
    size_t nk = (size_t)mx * mz * s->my;
    fld *lam = (fld *)malloc(sizeof(fld) * nk);
    /* cast x_sol -> lambda_3d (:1775-1781) */
#pragma omp parallel for
    for (ptrdiff_t q = 0; q < (ptrdiff_t)nk; q++) lam[q] = (fld)s->x[q];
#define LAM(i, k, j) lam[IK(s, (i), (k), (j))]
#define RHO(i, k, j) (adv_den ? d->density[IC(s, (i), (k), (j))] : (fld)1.0)
    /* rho_u / rho_v at one rank, :1818-1873 / :1875-1930; rho_w :1932-1946 */
    const fld *dz = d->advection_dz;
    fld dzk1 = s->dz_if[IZ(s, 1, 2, 1)], dzke = s->dz_if[IZ(s, 1, nz, 1)];
#pragma omp parallel for
    for (int j = 1; j <= ny; j++) {
        fld *ut = (fld *)malloc(sizeof(fld) * (size_t)(nx + 1) * (nz + 2));
        fld *udl = (fld *)malloc(sizeof(fld) * (size_t)(nx + 1) * nz);
#define UT(i, k) ut[(size_t)((i) - 1) + (size_t)(nx + 1) * (size_t)(k)]
#define UDL(i, k) udl[(size_t)((i) - 1) + (size_t)(nx + 1) * (size_t)((k) - 1)]
        for (int k = 0; k <= nz + 1; k++)
            for (int i = 1; i <= nx + 1; i++) UT(i, k) = (LAM(i, k, j) + LAM(i - 1, k, j)) / 2; /* :1948-1954 */
        for (int k = 1; k <= nz; k++) {
            fld den = s->dz_if[IZ(s, 1, k + 1, 1)] + s->dz_if[IZ(s, 1, k, 1)];
            for (int i = 1; i <= nx + 1; i++) { /* :1964-1970 */
                fld t = UT(i, k + 1) - UT(i, k - 1);
                UDL(i, k) = t / den;
            }
        }
        for (int i = 1; i <= nx + 1; i++) { /* one-sided :1984-1990 */
            UDL(i, 1) = (UT(i, 2) - UT(i, 1)) / dzk1;
            UDL(i, nz) = (UT(i, nz) - UT(i, nz - 1)) / dzke;
        }
        for (int k = 1; k <= nz; k++)
            for (int i = 1; i <= nx + 1; i++) { /* :2004-2013 */
                fld rho_u;
                if (i == 1) rho_u = RHO(1, k, j);
                else if (i == nx + 1) rho_u = RHO(nx, k, j);
                else rho_u = (fld)0.5 * (RHO(i, k, j) + RHO(i - 1, k, j));
                size_t q = IU(s, i, k, j);
                fld grad = (LAM(i, k, j) - LAM(i - 1, k, j)) / dx - d->dzdx_u[q] * (UDL(i, k)) / d->jacobian_u[q];
                u[q] = u[q] + (fld)0.5 * d->mapfac_mx_u[I2U(s, i, j)] * grad / (rho_u);
            }
        free(ut); free(udl);
#undef UT
#undef UDL
    }
#pragma omp parallel for
    for (int j = 1; j <= ny + 1; j++) {
        fld *vt = (fld *)malloc(sizeof(fld) * (size_t)nx * (nz + 2));
        fld *vdl = (fld *)malloc(sizeof(fld) * (size_t)nx * nz);
#define VT(i, k) vt[(size_t)((i) - 1) + (size_t)nx * (size_t)(k)]
#define VDL(i, k) vdl[(size_t)((i) - 1) + (size_t)nx * (size_t)((k) - 1)]
        for (int k = 0; k <= nz + 1; k++)
            for (int i = 1; i <= nx; i++) VT(i, k) = (LAM(i, k, j) + LAM(i, k, j - 1)) / 2; /* :1956-1962 */
        for (int k = 1; k <= nz; k++) {
            fld den = s->dz_if[IZ(s, 1, k + 1, 1)] + s->dz_if[IZ(s, 1, k, 1)];
            for (int i = 1; i <= nx; i++) { /* :1972-1978 */
                fld t = VT(i, k + 1) - VT(i, k - 1);
                VDL(i, k) = t / den;
            }
        }
        for (int i = 1; i <= nx; i++) { /* :1991-1997 */
            VDL(i, 1) = (VT(i, 2) - VT(i, 1)) / dzk1;
            VDL(i, nz) = (VT(i, nz) - VT(i, nz - 1)) / dzke;
        }
        for (int k = 1; k <= nz; k++)
            for (int i = 1; i <= nx; i++) { /* :2015-2024 */
                fld rho_v;
                if (j == 1) rho_v = RHO(i, k, 1);
                else if (j == ny + 1) rho_v = RHO(i, k, ny);
                else rho_v = (fld)0.5 * (RHO(i, k, j) + RHO(i, k, j - 1));
                size_t q = IV(s, i, k, j);
                fld grad = (LAM(i, k, j) - LAM(i, k, j - 1)) / dx - d->dzdy_v[q] * (VDL(i, k)) / d->jacobian_v[q];
                v[q] = v[q] + (fld)0.5 * d->mapfac_my_v[I2(s, i, j)] * grad / (rho_v);
            }
        free(vt); free(vdl);
#undef VT
#undef VDL
    }
    /* w_grid correction, rigid lid at k_e (:2038-2050) */
#pragma omp parallel for
    for (int j = 1; j <= ny; j++)
        for (int k = 1; k <= nz - 1; k++)
            for (int i = 1; i <= nx; i++) {
                size_t c = IC(s, i, k, j);
                fld rho_w;
                if (adv_den) {
                    size_t cp = IC(s, i, k + 1, j);
                    rho_w = (d->density[c] * dz[cp] + d->density[cp] * dz[c]) / (dz[c] + dz[cp]);
                } else rho_w = (fld)1.0;
                fld a = s->alpha[c];
                w[c] = w[c] + (fld)0.5 * (a * a) * (LAM(i, k + 1, j) - LAM(i, k, j)) / s->dz_if[IZ(s, i, k + 1, j)] / d->jacobian_w[c] / rho_w;
            }
#undef LAM
#undef RHO
    free(lam);
}

/* ------------------------------------------------------------------------ */
/* calc_divergence: wind.F90:250-523 (div(1:nx,1:nz,1:ny))                  */
/* ------------------------------------------------------------------------ */
void orc_calc_divergence(const orc_domain *d, const fld *u, const fld *v, const fld *w, fld *div,
                         int adv_den, int horz_only, int use_dqdt)
{
    orc_solver tmp; /* only for the index macros */
    tmp.nx = d->nx; tmp.ny = d->ny; tmp.nz = d->nz;
    orc_solver *s = &tmp;
    int nx = d->nx, ny = d->ny, nz = d->nz;
    fld dx = d->dx;
    const fld *rho = d->density, *ju = d->jacobian_u, *jv = d->jacobian_v, *jw = d->jacobian_w, *dz = d->advection_dz;
#pragma omp parallel for
    for (int j = 1; j <= ny; j++) {
        fld *um = (fld *)malloc(sizeof(fld) * (size_t)(nx + 1));
        fld *vm0 = (fld *)malloc(sizeof(fld) * (size_t)nx);
        fld *vm1 = (fld *)malloc(sizeof(fld) * (size_t)nx);
        fld *wm = (fld *)malloc(sizeof(fld) * (size_t)nx * nz);
        for (int k = 1; k <= nz; k++) {
            /* u_met over faces 1..nx+1 (:301-321 adv_den, :373-392 not) */
            for (int i = 1; i <= nx + 1; i++) {
                size_t q = IU(s, i, k, j);
                if (adv_den) {
                    if (i == 1) um[0] = u[q] * ju[q] * ((fld)1.5 * rho[IC(s, 1, k, j)] - (fld)0.5 * rho[IC(s, 2, k, j)]);
                    else if (i == nx + 1) um[nx] = u[q] * ju[q] * ((fld)1.5 * rho[IC(s, nx, k, j)] - (fld)0.5 * rho[IC(s, nx - 1, k, j)]);
                    else um[i - 1] = u[q] * ju[q] * (rho[IC(s, i - 1, k, j)] + rho[IC(s, i, k, j)]) / 2;
                } else um[i - 1] = use_dqdt ? u[q] : u[q] * ju[q];
            }
            /* v_met for faces j and j+1 of this row */
            for (int jj = 0; jj < 2; jj++) {
                int jf = j + jj;
                fld *vm = jj ? vm1 : vm0;
                for (int i = 1; i <= nx; i++) {
                    size_t q = IV(s, i, k, jf);
                    if (adv_den) {
                        if (jf == 1) vm[i - 1] = v[q] * jv[q] * ((fld)1.5 * rho[IC(s, i, k, 1)] - (fld)0.5 * rho[IC(s, i, k, 2)]);
                        else if (jf == ny + 1) vm[i - 1] = v[q] * jv[q] * ((fld)1.5 * rho[IC(s, i, k, ny)] - (fld)0.5 * rho[IC(s, i, k, ny - 1)]);
                        else vm[i - 1] = v[q] * jv[q] * (rho[IC(s, i, k, jf - 1)] + rho[IC(s, i, k, jf)]) / 2;
                    } else vm[i - 1] = use_dqdt ? v[q] : v[q] * jv[q];
                }
            }
            /* horizontal divergence with map factors (:400-409) */
            for (int i = 1; i <= nx; i++) {
                fld sum = um[i] / d->mapfac_my_u[I2U(s, i + 1, j)] - um[i - 1] / d->mapfac_my_u[I2U(s, i, j)] +
                          vm1[i - 1] / d->mapfac_mx_v[I2(s, i, j + 1)] - vm0[i - 1] / d->mapfac_mx_v[I2(s, i, j)];
                div[IC(s, i, k, j)] = d->mapfac_mxy[I2(s, i, j)] * sum / dx;
            }
        }
        if (!horz_only) {
            /* w_met (:411-466) */
            for (int k = 1; k <= nz; k++)
                for (int i = 1; i <= nx; i++) {
                    size_t c = IC(s, i, k, j);
                    fld wv;
                    if (adv_den) {
                        if (k < nz) {
                            size_t cp = IC(s, i, k + 1, j);
                            fld rho_i = (rho[c] * dz[cp] + rho[cp] * dz[c]) / (dz[c] + dz[cp]); /* :355-361 */
                            wv = w[c] * jw[c] * rho_i;
                        } else wv = w[c] * jw[c] * rho[c];
                    } else wv = w[c] * jw[c];
                    wm[(size_t)(i - 1) + (size_t)nx * (k - 1)] = wv;
                }
            /* vertical flux difference and jacobian (:468-482) */
            for (int k = 1; k <= nz; k++)
                for (int i = 1; i <= nx; i++) {
                    size_t c = IC(s, i, k, j);
                    fld dv = div[c];
                    if (k == 1) dv = dv + wm[(size_t)(i - 1)] / (dz[c]);
                    else dv = dv + (wm[(size_t)(i - 1) + (size_t)nx * (k - 1)] - wm[(size_t)(i - 1) + (size_t)nx * (k - 2)]) / (dz[c]);
                    dv = dv / d->jacobian[c];
                    div[c] = dv;
                }
        }
        free(um); free(vm0); free(vm1); free(wm);
    }
}

/* ------------------------------------------------------------------------ */
/* solver object                                                            */
/* ------------------------------------------------------------------------ */
orc_solver *orc_create(const orc_domain *d, int max_iters)
{
    orc_solver *s = (orc_solver *)calloc(1, sizeof(orc_solver));
    s->d = *d;
    s->nx = d->nx; s->ny = d->ny; s->nz = d->nz;
    s->mx = d->nx + 2; s->my = d->ny + 2; s->mz = d->nz + 2;
    s->dx = d->dx;
    s->ncell = (size_t)d->nx * d->nz * d->ny;
    s->nrows = (size_t)s->mx * s->my * s->mz;
    s->dz_if = (fld *)calloc((size_t)d->nx * (d->nz + 1) * d->ny, sizeof(fld));
    s->dzdx_surf = (fld *)calloc((size_t)d->nx * d->ny, sizeof(fld));
    s->dzdy_surf = (fld *)calloc((size_t)d->nx * d->ny, sizeof(fld));
    s->adv_dz_col = (fld *)calloc((size_t)d->nz, sizeof(fld));
    s->alpha = (fld *)calloc(s->ncell, sizeof(fld));
    s->div = (fld *)calloc(s->ncell, sizeof(fld));
    for (int c = 0; c < NCOEF; c++) s->coef[c] = (fld *)calloc(s->ncell, sizeof(fld));
    double **vecs[] = {&s->x, &s->r, &s->rhat, &s->p, &s->phat, &s->v, &s->s, &s->shat, &s->t, &s->rhs, &s->Dinv, &s->pres};
    for (size_t q = 0; q < sizeof(vecs) / sizeof(vecs[0]); q++) *vecs[q] = (double *)calloc(s->nrows, sizeof(double));
    s->max_iters = max_iters > 0 ? max_iters : 1500; /* namelist default, namelist_utilities.F90:3871-3876 */
    s->tol_rel = 1.0e-5;                              /* wind_iterative.F90:60 */
    s->tol_abs = 1.0e-10;                             /* wind_iterative.F90:59 */
    s->precond_n_sweeps = BASE_PREC_SWEEPS;
    init_module_vars(s);
    return s;
}

void orc_destroy(orc_solver *s)
{
    if (!s) return;
    free(s->dz_if); free(s->dzdx_surf); free(s->dzdy_surf); free(s->adv_dz_col); free(s->alpha); free(s->div);
    for (int c = 0; c < NCOEF; c++) free(s->coef[c]);
    double *vecs[] = {s->x, s->r, s->rhat, s->p, s->phat, s->v, s->s, s->shat, s->t, s->rhs, s->Dinv, s->pres};
    for (size_t q = 0; q < sizeof(vecs) / sizeof(vecs[0]); q++) free(vecs[q]);
    free(s->hist);
    free(s);
}

void orc_set_tolerance(orc_solver *s, double tol_rel, double tol_abs)
{
    s->tol_rel = tol_rel;
    s->tol_abs = tol_abs;
}

/* calc_iter_winds: wind_iterative.F90:295-532.  Returns 0, or -1 where the
 * reference executes `stop` (diverged after every retry, :506-528); the
 * corrected winds are written into u, v, w. */
int orc_calc_iter_winds(orc_solver *s, const fld *alpha_in, const fld *div_in, int adv_den, fld *u, fld *v, fld *w, orc_stats *out)
{
    orc_stats st;
    memset(&st, 0, sizeof(st));
    memcpy(s->div, div_in, s->ncell * sizeof(fld));     /* :308-317 */
    memcpy(s->alpha, alpha_in, s->ncell * sizeof(fld));
    if (!s->structure_uploaded) {                        /* :351-407 */
        initialize_coefs(s);
        vec_zero(s, s->x);
        s->structure_uploaded = 1;
    } else {                                              /* :408-427 */
        fld amin = s->alpha[0], amax = s->alpha[0];
        for (size_t q = 0; q < s->ncell; q++) {
            if (s->alpha[q] < amin) amin = s->alpha[q];
            if (s->alpha[q] > amax) amax = s->alpha[q];
        }
        if (amax > amin && !s->operator_probed) update_coefs_gpu(s);
    }
    extract_diagonal(s);                                  /* :430 */
    compute_rhs_3d(s);                                    /* :433 */
    orc_bicgstab(s, s->max_iters, &st);                   /* :445, warm start from x_sol */
    st.sweeps = s->precond_n_sweeps;
    double res0_first = st.res0;
    (void)res0_first;
    if (st.status != 0 && st.iters > 0 && st.res_final > 0.01 * st.res0) { /* :479-503 */
        while (st.status != 0 && st.res_final > 0.01 * st.res0 && s->precond_n_sweeps < MAX_PREC_SWEEPS) {
            s->precond_n_sweeps++;
            vec_zero(s, s->x);
            int retries = st.retries + 1;
            orc_bicgstab(s, s->max_iters, &st);
            st.retries = retries;
            st.sweeps = s->precond_n_sweeps;
        }
        s->precond_n_sweeps = BASE_PREC_SWEEPS;          /* :504 */
        if (st.status != 0 && st.res_final > st.res0) {  /* :506-528 -> `stop` */
            st.fatal = 1;
            s->last = st;
            if (out) *out = st;
            return -1;
        }
    }
    orc_calc_updated_winds(s, adv_den, u, v, w);          /* :531 */
    s->last = st;
    if (out) *out = st;
    return 0;
}

/* ---- probing: wind_iterative.F90:1096-1248, orchestrated by wind.F90:1010-1099 ---- */
void orc_probe_lambda_pattern(orc_solver *s, int ca, int cb, int cc)
{
    int mx = s->mx, my = s->my, mz = s->mz;
#pragma omp parallel for
    for (int j = 0; j < my; j++)
        for (int k = 0; k < mz; k++)
            for (int i = 0; i < mx; i++) {
                int on = i >= 1 && i <= mx - 2 && k >= 1 && k <= mz - 2 && j >= 1 && j <= my - 2 && i % 3 == ca && k % 3 == cb && j % 3 == cc;
                s->x[IK(s, i, k, j)] = on ? 1.0 : 0.0;
            }
}

void orc_probe_record(orc_solver *s, const fld *Tfield, int ca, int cb, int cc, fld *max_leak)
{
    int nx = s->nx, ny = s->ny, nz = s->nz;
    fld leak = *max_leak;
    for (int j = 1; j <= ny; j++)
        for (int k = 1; k <= nz; k++)
            for (int i = 1; i <= nx; i++) {
                int di = (ca - i % 3 + 3) % 3; if (di == 2) di = -1;
                int dk = (cb - k % 3 + 3) % 3; if (dk == 2) dk = -1;
                int dj = (cc - j % 3 + 3) % 3; if (dj == 2) dj = -1;
                size_t c = IC(s, i, k, j);
                fld tv = (fld)2.0 * Tfield[c];
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
                if (slot >= 0) s->coef[slot][c] = tv;
                else if (fabs((double)tv) > (double)leak) leak = (fld)fabs((double)tv);
            }
    *max_leak = leak;
}

void orc_probe_finalize(orc_solver *s)
{
    s->operator_probed = 1;
    vec_zero(s, s->x);
}

/* calibrate_projection_operator: wind.F90:1010-1099.  u, v, w are the caller's
 * dqdt winds; they are saved, used as probe scratch and restored. */
fld orc_calibrate(orc_solver *s, int adv_den, fld *u, fld *v, fld *w)
{
    int nx = s->nx, ny = s->ny, nz = s->nz;
    size_t nu = (size_t)(nx + 1) * nz * ny, nv = (size_t)nx * nz * (ny + 1), nw = (size_t)nx * nz * ny;
    fld *us = (fld *)malloc(nu * sizeof(fld)), *vs = (fld *)malloc(nv * sizeof(fld)), *ws = (fld *)malloc(nw * sizeof(fld));
    fld *div = (fld *)malloc(nw * sizeof(fld));
    memcpy(us, u, nu * sizeof(fld)); memcpy(vs, v, nv * sizeof(fld)); memcpy(ws, w, nw * sizeof(fld));
    fld max_leak = 0;
    for (int cc = 0; cc < 3; cc++)
        for (int cb = 0; cb < 3; cb++)
            for (int ca = 0; ca < 3; ca++) {
                orc_probe_lambda_pattern(s, ca, cb, cc);
                memset(u, 0, nu * sizeof(fld)); memset(v, 0, nv * sizeof(fld)); memset(w, 0, nw * sizeof(fld));
                orc_calc_updated_winds(s, adv_den, u, v, w);
                orc_calc_divergence(&s->d, u, v, w, div, adv_den, 0, 1);
                orc_probe_record(s, div, ca, cb, cc, &max_leak);
            }
    orc_probe_finalize(s);
    memcpy(u, us, nu * sizeof(fld)); memcpy(v, vs, nv * sizeof(fld)); memcpy(w, ws, nw * sizeof(fld));
    free(us); free(vs); free(ws); free(div);
    return max_leak;
}

/* ---- accessors used by the tests ---- */
void orc_build_analytic(orc_solver *s, const fld *alpha_in)
{
    memcpy(s->alpha, alpha_in, s->ncell * sizeof(fld));
    initialize_coefs(s);
    s->structure_uploaded = 1;
}
void orc_refresh_coefs(orc_solver *s, const fld *alpha_in)
{
    memcpy(s->alpha, alpha_in, s->ncell * sizeof(fld));
    update_coefs_gpu(s);
}
void orc_prepare_solve(orc_solver *s, const fld *div_in)
{
    memcpy(s->div, div_in, s->ncell * sizeof(fld));
    extract_diagonal(s);
    compute_rhs_3d(s);
}
void orc_set_alpha(orc_solver *s, const fld *alpha_in) { memcpy(s->alpha, alpha_in, s->ncell * sizeof(fld)); }
void orc_get_coefs(orc_solver *s, int which, fld *out) { memcpy(out, s->coef[which], s->ncell * sizeof(fld)); }
void orc_set_coefs(orc_solver *s, int which, const fld *in) { memcpy(s->coef[which], in, s->ncell * sizeof(fld)); }
void orc_set_probed(orc_solver *s, int probed) { s->operator_probed = probed; s->structure_uploaded = 1; }
void orc_get_vec(orc_solver *s, int which, double *out)
{
    double *v[] = {s->x, s->r, s->rhat, s->p, s->phat, s->v, s->s, s->shat, s->t, s->rhs, s->Dinv, s->pres};
    memcpy(out, v[which], s->nrows * sizeof(double));
}
void orc_set_vec(orc_solver *s, int which, const double *in)
{
    double *v[] = {s->x, s->r, s->rhat, s->p, s->phat, s->v, s->s, s->shat, s->t, s->rhs, s->Dinv, s->pres};
    memcpy(v[which], in, s->nrows * sizeof(double));
}
void orc_set_sweeps(orc_solver *s, int n) { s->precond_n_sweeps = n; }
void orc_set_max_iters(orc_solver *s, int n) { s->max_iters = n; }
int orc_get_hist(orc_solver *s, double *out, int cap)
{
    int n = s->hist_len < cap ? s->hist_len : cap;
    if (out) memcpy(out, s->hist, (size_t)n * sizeof(double));
    return s->hist_len;
}
void orc_get_stats(orc_solver *s, orc_stats *out) { *out = s->last; }
void orc_get_surf(orc_solver *s, fld *dzdx_surf, fld *dzdy_surf, fld *dz_if)
{
    memcpy(dzdx_surf, s->dzdx_surf, (size_t)s->nx * s->ny * sizeof(fld));
    memcpy(dzdy_surf, s->dzdy_surf, (size_t)s->nx * s->ny * sizeof(fld));
    memcpy(dz_if, s->dz_if, (size_t)s->nx * (s->nz + 1) * s->ny * sizeof(fld));
}
/* true residual ||b - A x|| in FP64 over all rows */
double orc_true_residual(orc_solver *s)
{
    orc_spmv(s, s->x, s->pres);
    double acc = 0.0;
    for (size_t q = 0; q < s->nrows; q++) {
        double e = s->rhs[q] - s->pres[q];
        acc += e * e;
    }
    return sqrt(acc);
}

/* ------------------------------------------------------------------------ */
/* the steps either side of the solve in update_winds (wind.F90)            */
/* ------------------------------------------------------------------------ */

/* calc_w_real (wind.F90:1175-1227): w_real = mean of u dz/dx over the two
 * u faces + mean of v dz/dy over the two v faces + mean of w_grid * jaco over
 * the two w levels (zero below the first), jaco = jacobian_w.  w_grid may be
 * NULL (all zero, as calc_idealized_wgrid passes it). */
void orc_calc_w_real(const orc_domain *d, const fld *u, const fld *v, const fld *w_grid, fld *w_real)
{
    orc_solver tmp;
    tmp.nx = d->nx; tmp.ny = d->ny; tmp.nz = d->nz;
    orc_solver *s = &tmp;
    const fld *jw = d->jacobian_w;
#pragma omp parallel for
    for (int j = 1; j <= d->ny; j++)
        for (int k = 1; k <= d->nz; k++)
            for (int i = 1; i <= d->nx; i++) {
                size_t c = IC(s, i, k, j);
                fld lo = 0, hi = 0;
                if (w_grid) {
                    hi = w_grid[c] * jw[c];
                    if (k > 1) lo = w_grid[IC(s, i, k - 1, j)] * jw[IC(s, i, k - 1, j)];
                }
                w_real[c] = (u[IU(s, i, k, j)] * d->dzdx_u[IU(s, i, k, j)] + u[IU(s, i + 1, k, j)] * d->dzdx_u[IU(s, i + 1, k, j)]) * (fld)0.5
                          + (v[IV(s, i, k, j)] * d->dzdy_v[IV(s, i, k, j)] + v[IV(s, i, k, j + 1)] * d->dzdy_v[IV(s, i, k, j + 1)]) * (fld)0.5
                          + (lo + hi) * (fld)0.5;
            }
}

/* calc_idealized_wgrid (wind.F90:940-998): w = w_real_field - calc_w_real(u, v, 0),
 * staggered to the w levels with advection_dz weights, divided by jacobian_w,
 * zero at the top level. */
void orc_calc_idealized_wgrid(const orc_domain *d, const fld *u, const fld *v, const fld *w_real_field, fld *w)
{
    orc_solver tmp;
    tmp.nx = d->nx; tmp.ny = d->ny; tmp.nz = d->nz;
    orc_solver *s = &tmp;
    const fld *dz = d->advection_dz, *jw = d->jacobian_w;
    orc_calc_w_real(d, u, v, NULL, w);
    size_t n = (size_t)d->nx * d->nz * d->ny;
    for (size_t q = 0; q < n; q++) w[q] = w_real_field[q] - w[q];
#pragma omp parallel for
    for (int j = 1; j <= d->ny; j++)
        for (int i = 1; i <= d->nx; i++) {
            for (int k = 1; k <= d->nz - 1; k++) { /* w(k+1) still holds its unstaggered value */
                size_t c = IC(s, i, k, j), cp = IC(s, i, k + 1, j);
                w[c] = (w[c] * dz[cp] + w[cp] * dz[c]) / (dz[c] + dz[cp]);
                w[c] = w[c] / jw[c];
            }
            w[IC(s, i, d->nz, j)] = 0;
        }
}

/* calc_w (wind.F90:201-248): w integrated upward from a (horizontal) divergence. */
void orc_calc_w(const orc_domain *d, fld *w, const fld *div, int adv_den)
{
    orc_solver tmp;
    tmp.nx = d->nx; tmp.ny = d->ny; tmp.nz = d->nz;
    orc_solver *s = &tmp;
    const fld *dz = d->advection_dz, *jw = d->jacobian_w, *rho = d->density;
    int nz = d->nz;
#pragma omp parallel for
    for (int j = 1; j <= d->ny; j++)
        for (int i = 1; i <= d->nx; i++) {
            fld rho_prev = 0;
            for (int k = 1; k <= nz; k++) {
                size_t c = IC(s, i, k, j);
                fld rho_i = 0;
                if (adv_den) {
                    if (k < nz) {
                        size_t cp = IC(s, i, k + 1, j);
                        rho_i = (rho[c] * dz[cp] + rho[cp] * dz[c]) / (dz[c] + dz[cp]);
                    } else rho_i = rho[c];
                    if (k == 1) w[c] = 0 - div[c] * dz[c] / (jw[c] * rho_i);
                    else {
                        size_t cm = IC(s, i, k - 1, j);
                        w[c] = ((w[cm] * rho_prev * jw[cm]) - div[c] * dz[c]) / (jw[c] * rho_i);
                    }
                } else {
                    if (k == 1) w[c] = (0 - div[c] * dz[c]) / (jw[c]);
                    else {
                        size_t cm = IC(s, i, k - 1, j);
                        w[c] = (w[cm] * jw[cm] - div[c] * dz[c]) / (jw[c]);
                    }
                }
                rho_prev = rho_i;
            }
        }
}

/* balance_uvw (wind.F90:123-199): w from the horizontal divergence of u, v. */
void orc_balance_uvw(const orc_domain *d, const fld *u, const fld *v, fld *w, int adv_den, int use_dqdt)
{
    size_t n = (size_t)d->nx * d->nz * d->ny;
    fld *div = (fld *)malloc(n * sizeof(fld));
    orc_calc_divergence(d, u, v, w, div, adv_den, 1, use_dqdt);
    orc_calc_w(d, w, div, adv_den);
    free(div);
}

/* calc_alpha (wind.F90:1102-1173): alpha from the Froude number (Moussiopoulos
 * et al. 1988), bounded to [0.2, 2], 0.2 on the top level, and the `halo`
 * outermost rows/columns copied from the first tile row/column (south, west,
 * north, east, in that order).  (1/Fr)**4 is evaluated as (t*t)*(t*t). */
void orc_calc_alpha(int nx, int ny, int nz, const fld *froude, fld *alpha, int halo)
{
    const fld amin = (fld)0.2, amax = (fld)2.0;
    size_t n = (size_t)nx * nz * ny;
    for (size_t q = 0; q < n; q++) {
        fld t = (fld)1.0 / froude[q];
        fld t2 = t * t;
        fld p = t2 * t2;
        fld mx = p > (fld)0.00001 ? p : (fld)0.00001;
        fld a = (fld)1.0 - (fld)0.5 * mx * (FLD_SQRT((fld)1.0 + (fld)4.0 / mx) - (fld)1.0);
        a = FLD_SQRT(a > (fld)0.00001 ? a : (fld)0.00001);
        a = a > amin ? a : amin;
        a = a < amax ? a : amax;
        alpha[q] = a;
    }
#define IA(i, k, j) ((size_t)((i) - 1) + (size_t)nx * ((size_t)((k) - 1) + (size_t)nz * (size_t)((j) - 1)))
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) alpha[IA(i, nz, j)] = amin;
    if (halo > 0) {
        for (int j = 1; j <= halo; j++)
            for (int k = 1; k <= nz; k++)
                for (int i = 1; i <= nx; i++) alpha[IA(i, k, j)] = alpha[IA(i, k, halo + 1)];
        for (int j = 1; j <= ny; j++)
            for (int k = 1; k <= nz; k++)
                for (int i = 1; i <= halo; i++) alpha[IA(i, k, j)] = alpha[IA(halo + 1, k, j)];
        for (int j = ny - halo + 1; j <= ny; j++)
            for (int k = 1; k <= nz; k++)
                for (int i = 1; i <= nx; i++) alpha[IA(i, k, j)] = alpha[IA(i, k, ny - halo)];
        for (int j = 1; j <= ny; j++)
            for (int k = 1; k <= nz; k++)
                for (int i = nx - halo + 1; i <= nx; i++) alpha[IA(i, k, j)] = alpha[IA(nx - halo, k, j)];
    }
#undef IA
}

/* smooth_array_3d with ydim = 3 (array_utilities.F90:322-397), `nsmooths`
 * passes: each level's x-y field replaced by its (2w+1)^2 box mean with
 * edge-replicated (clamped) indices, summed in double (y offset outer, x inner)
 * from the values before the pass. */
void orc_smooth_array(int nx, int ny, int nz, fld *a, int window, int nsmooths)
{
    size_t n = (size_t)nx * nz * ny;
    fld *in = (fld *)malloc(n * sizeof(fld));
    const int nc = window * 2 + 1;
    for (int pass = 0; pass < nsmooths; pass++) {
        memcpy(in, a, n * sizeof(fld));
#pragma omp parallel for
        for (int j = 1; j <= ny; j++)
            for (int k = 1; k <= nz; k++)
                for (int i = 1; i <= nx; i++) {
                    double cur = 0.0;
                    for (int dj = -window; dj <= window; dj++) {
                        int jj = j + dj < 1 ? 1 : (j + dj > ny ? ny : j + dj);
                        for (int di = -window; di <= window; di++) {
                            int ii = i + di < 1 ? 1 : (i + di > nx ? nx : i + di);
                            cur = cur + (double)in[(size_t)(ii - 1) + (size_t)nx * ((size_t)(k - 1) + (size_t)nz * (jj - 1))];
                        }
                    }
                    a[(size_t)(i - 1) + (size_t)nx * ((size_t)(k - 1) + (size_t)nz * (j - 1))] = (fld)(cur / (double)(nc * nc));
                }
    }
    free(in);
}

/* ------------------------------------------------------------------------ */
/* update_stability (wind.F90:1421-1565) with its helpers calc_dry_stability,  */
/* calc_Ri and calc_froude (atm_utilities.F90:466-546)                       */
/* ------------------------------------------------------------------------ */
#define ORC_GRAVITY ((fld)9.81)          /* mod_wrf_constants gravity */
#define ORC_RAD2DEG ((fld)57.2957779371) /* wind.F90:39 */
#if defined(ORC_FLD_DOUBLE)
#define FLD_ATAN2 atan2
#else
#define FLD_ATAN2 atan2f
#endif

/* calc_dry_stability (atm_utilities.F90:466-479); has_surf selects the th_surf form */
static fld orc_dry_stability(fld th_top, fld th_bot, fld z_top, fld z_bot, int has_surf, fld th_surf)
{
    if (has_surf) return ORC_GRAVITY * (th_top - th_bot) / ((z_top - z_bot) * th_surf);
    return ORC_GRAVITY * (th_top - th_bot) / ((z_top - z_bot) * (th_top + th_bot) / (fld)2);
}

/* calc_Ri (atm_utilities.F90:528-546) */
static fld orc_calc_ri(fld bv2, fld u_shear, fld v_shear, fld dz)
{
    fld a = u_shear / dz, b = v_shear / dz;
    fld denom = a * a + b * b;
    return denom == (fld)0 ? (fld)10 : bv2 / denom;
}

/* calc_froude (atm_utilities.F90:504-525) */
static fld orc_calc_froude(fld bv2, fld barrier_height, fld wind_speed)
{
    fld n = FLD_SQRT(bv2 > (fld)0 ? bv2 : (fld)0);
    fld denom = barrier_height * n;
    return denom == (fld)0 ? (fld)100 : wind_speed / denom;
}

/* update_stability at one rank: u (nx+1, nz, ny), v (nx, nz, ny+1) are the dqdt
 * winds, z and theta (nx, nz, ny) the mass-level heights and potential
 * temperature, froude_terrain (nx, nz, ny, nsect) the blocking heights per
 * 5-degree wind-direction sector.  Writes froude and blk_ri (nx, nz, ny);
 * froude_mode != 0 is the branch of alpha_const < 0 with iterative winds
 * (otherwise froude stays 0.1). */
void orc_update_stability(int nx, int ny, int nz, const fld *u, const fld *v, const fld *z, const fld *theta,
                          const fld *froude_terrain, int nsect, int froude_mode, fld *froude, fld *blk_ri)
{
    const fld RI_Z_MAX = (fld)100.0;
#define SC(i, k, j) ((size_t)((i) - 1) + (size_t)nx * ((size_t)((k) - 1) + (size_t)nz * (size_t)((j) - 1)))
#define SU(i, k, j) ((size_t)((i) - 1) + (size_t)(nx + 1) * ((size_t)((k) - 1) + (size_t)nz * (size_t)((j) - 1)))
#define SV(i, k, j) ((size_t)((i) - 1) + (size_t)nx * ((size_t)((k) - 1) + (size_t)nz * (size_t)((j) - 1)))
#pragma omp parallel for
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            int rk = nz; /* Ri_k_max (:1444-1454) */
            for (int k = 2; k <= nz; k++)
                if (z[SC(i, k, j)] - z[SC(i, 1, j)] > RI_Z_MAX) {
                    rk = k - 1 > 2 ? k - 1 : 2;
                    break;
                }
            /* u_m, v_m (:1457-1460) and the surface shear u_m(:, kms+4, :) (:1462-1465) */
            fld us = (u[SU(i, 5, j)] + u[SU(i + 1, 5, j)]) / (fld)2;
            fld vs = (v[SV(i, 5, j)] + v[SV(i, 5, j + 1)]) / (fld)2;
            for (int k = 1; k <= nz; k++) { /* (:1472-1480) */
                froude[SC(i, k, j)] = (fld)0.1;
                blk_ri[SC(i, k, j)] = (fld)10.0;
            }
            for (int k = 1; k <= nz - 1; k++) { /* (:1482-1495) */
                fld th_bot = theta[SC(i, 1, j)], th_top = theta[SC(i, rk, j)];
                fld z_bot = z[SC(i, 1, j)], z_top = z[SC(i, rk, j)];
                fld stab = orc_dry_stability(th_top, th_bot, z_top, z_bot, 0, (fld)0);
                blk_ri[SC(i, k, j)] = orc_calc_ri(stab, us, vs, z_top - z_bot);
            }
            if (!froude_mode) continue;
            for (int k = 1; k <= nz - 1; k++) { /* (:1503-1560) */
                fld um = (u[SU(i, k, j)] + u[SU(i + 1, k, j)]) / (fld)2;
                fld vm = (v[SV(i, k, j)] + v[SV(i, k, j + 1)]) / (fld)2;
                fld ws = FLD_SQRT(um * um + vm * vm);
                fld wd = FLD_ATAN2(-um, -vm) * ORC_RAD2DEG;
                if (wd <= (fld)0.0) wd = wd + (fld)360;
                if (wd == (fld)360.0) wd = (fld)0.0;
                int dir = (int)(wd / (fld)5) + 1;
                dir = dir < nsect ? dir : nsect;
                dir = dir > 1 ? dir : 1;
                fld tf = froude_terrain[SC(i, k, j) + (size_t)(dir - 1) * (size_t)nx * nz * ny];
                fld stab = orc_dry_stability(theta[SC(i, k + 1, j)], theta[SC(i, k, j)], z[SC(i, k + 1, j)],
                                             z[SC(i, k, j)], 1, theta[SC(i, 1, j)]);
                froude[SC(i, k, j)] = orc_calc_froude(stab, tf, ws);
            }
        }
#undef SC
#undef SU
#undef SV
}
