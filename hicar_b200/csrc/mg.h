// mg.h -- multigrid V-cycle preconditioner (k_mg.cu).
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace hw {

constexpr int MG_MAX_LEVELS = 16;

struct MgLevel {
    Dims d;
    const float *coef = nullptr; // 15 * npad (level 0: the solver's probed coefficients)
    float *cp = nullptr;         // Thomas factors of the column tridiagonal
    float *minv = nullptr;
    float *r = nullptr;          // level right-hand side (levels >= 1)
    float *x1 = nullptr;         // pre-smoothed iterate
    float *x3 = nullptr;         // post-smoothed iterate (levels >= 1)
};

struct Mg {
    int nlev = 0;
    int ready = 0;
    float omega = 0.8f;  // damping of the z-line Jacobi smoother
    float cscale = 1.0f; // scale of the prolongated coarse-grid correction (over-correction > 1)
    int pre0 = 1;        // pre-smooth the finest level (0: V(0,1) there, its x1 kept at zero)
    int wmask = 0;       // bit l (l >= 1): level l corrects twice from the coarse grid (W-cycle there)
    int use_tma = 2;     // post-smoothers of the wide levels: 2 tensor copies, recurrences on their own warp
                         // (post_tma2_kernel); 1 tensor copies, post_tma_kernel (HICARW_MG_TMA=1);
                         // 0 register-fed (HICARW_MG_TMA=0)
    int fuse_level = 0;  // first level of the coarse part run by one thread-block cluster (0: every level its own
                         // launches; HICARW_MG_FUSE=0 at build time)
    int cluster_n = 0;   // CTAs of that cluster
    int bf16 = 0;        // the finest level's smoother coefficients in BF16 (V(0,1) cycles; factors of the rounded
                         // tridiagonal)
    __nv_bfloat16 *coef0h = nullptr; // those coefficients (15 * npad)
    int *err = nullptr;  // device flag: a bounded copy wait of a smoother timed out (calls without a solve state)
    MgLevel lev[MG_MAX_LEVELS];
};

int mg_build(Mg &mg, const Dims &fine, const float *fine_coef, cudaStream_t s);
void mg_free(Mg &mg);
long long mg_tma_posts(); // post-smoother launches enqueued through the tensor-copy kernel
template <typename V>
void mg_apply(const Mg &mg, const V *in, V *out, const SolveState *gate, cudaStream_t s);
// one bounded mbarrier wait that nothing completes, limit_ns long; sets *err on time-out
void mg_wait_probe(int *err, uint64_t limit_ns, cudaStream_t s);
template <typename V>
void launch_s_update(const Dims &d, const V *r, const V *v, V *s, const SolveState *stt, cudaStream_t st);

}  // namespace hw
