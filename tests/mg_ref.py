"""CPU restatement (numpy) of the multigrid V-cycle preconditioner of
hicar_b200/csrc/k_mg.cu, used by the GPU tests as the checker of that kernel
set.  The V-cycle has no counterpart in the reference; this restates the same
algorithm with the same FP32 storage points:
  * 2x2 x-y aggregation, Galerkin coarse operator (FP64 sums stored in FP32),
    couplings to cells outside the interior dropped, down to one column;
  * z-line Jacobi smoother with the column tridiagonal (C, A, B): Thomas
    factors computed in FP64 and stored in FP32, the recurrences in FP32, the
    residual of the post-smoother summed in FP64 from the FP32 staged iterate
    x2 = x1 + cscale P xc (FP32, cscale the over-correction), damping omega;
    exact tridiagonal solve on the
    single-column level (reached by the fused restriction + pre-smoothing).
Arrays are the interior (ny, nz, nx) blocks; coefficients are (15, ny, nz, nx)
in the order A..O.
"""
import numpy as np

# offsets (dk, dj, di) of A..O
OFF = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 1), (1, 0, -1),
       (-1, 0, 1), (-1, 0, -1), (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0)]
SLOT = {o: q for q, o in enumerate(OFF)}
f32 = np.float32


def shift(x, dk, dj, di):
    """y[j, k, i] = x[j+dj, k+dk, i+di], zero outside."""
    y = np.zeros_like(x)
    ny, nz, nx = x.shape

    def sl(n, d):
        return slice(max(0, d), n + min(0, d)), slice(max(0, -d), n - max(0, d))

    (sj, dj2), (sk, dk2), (si, di2) = sl(ny, dj), sl(nz, dk), sl(nx, di)
    y[dj2, dk2, di2] = x[sj, sk, si]
    return y


def apply(C, x):
    y = np.zeros(x.shape, np.float64)
    for q, (dk, dj, di) in enumerate(OFF):
        y += C[q].astype(np.float64) * shift(x.astype(np.float64), dk, dj, di)
    return y


def coarsen(C):
    _, ny, nz, nx = C.shape
    nyc, nxc = (ny + 1) // 2, (nx + 1) // 2
    Cc = np.zeros((15, nyc, nz, nxc), np.float64)
    kk = np.arange(nz)
    for q, (dk, dj, di) in enumerate(OFF):
        for pj in (0, 1):
            for pi in (0, 1):
                sub = C[q][pj::2, :, pi::2].astype(np.float64)
                jf = np.arange(pj, ny, 2)[:, None, None]
                if_ = np.arange(pi, nx, 2)[None, None, :]
                k3 = kk[None, :, None]
                ok = (jf + dj >= 0) & (jf + dj < ny) & (if_ + di >= 0) & (if_ + di < nx) & \
                     (k3 + dk >= 0) & (k3 + dk < nz)
                cdj = (pj + dj) // 2
                cdi = (pi + di) // 2
                q2 = SLOT[(dk, cdj, cdi)]
                Cc[q2, :sub.shape[0], :, :sub.shape[2]] += np.where(ok, sub, 0.0)
    return Cc.astype(f32)


def factors(C):
    A, B, Cs = C[0].astype(np.float64), C[1].astype(np.float64), C[2].astype(np.float64)
    nz = A.shape[1]
    cp = np.zeros(A.shape, np.float64)
    mi = np.zeros(A.shape, np.float64)
    cprev = np.zeros(A[:, 0].shape)
    for k in range(nz):
        a = Cs[:, k] if k > 0 else 0.0
        c = B[:, k] if k < nz - 1 else 0.0
        den = A[:, k] - a * cprev
        m = 1.0 / den
        mi[:, k] = m
        cprev = c * m
        cp[:, k] = cprev
    return cp.astype(f32), mi.astype(f32)


def thomas32(C, cp, mi, res):
    """T^-1 res column by column, FP32 recurrences (couplings to ghost planes dropped)."""
    nz = res.shape[1]
    d = np.zeros(res.shape, f32)
    dprev = np.zeros(res[:, 0].shape, f32)
    for k in range(nz):
        a = C[2][:, k] if k > 0 else f32(0)
        dv = ((res[:, k] - a * dprev) * mi[:, k]).astype(f32)
        d[:, k] = dv
        dprev = dv
    y = np.zeros(res[:, 0].shape, f32)
    for k in range(nz - 1, -1, -1):
        y = (d[:, k] - cp[:, k] * y).astype(f32)
        d[:, k] = y
    return d


def pre(C, cp, mi, r, omega):
    """out = omega T^-1 r (from zero)."""
    return (f32(omega) * thomas32(C, cp, mi, np.asarray(r).astype(f32))).astype(f32)


def post(C, cp, mi, r, x2, omega):
    """out = x2 + omega T^-1 (r - A x2), x2 given in FP32."""
    res = (np.asarray(r, np.float64) - apply(C, x2)).astype(f32)
    y = thomas32(C, cp, mi, res)
    return x2.astype(np.float64) + float(omega) * y.astype(np.float64)


def bf16_round(a):
    """FP32 values rounded to the nearest BF16 (ties to even), kept as FP32."""
    u = np.asarray(a, f32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(f32)


class VCycle:
    """fine_presmooth=False: V(0,1) on the finest level (its x1 is zero, level 1
    restricts the input itself).  wlevels: levels (>= 1) that correct twice from
    their coarse grid per visit (W-cycle there): the second restriction takes the
    residual of the first post-smoothed iterate, stored in FP32 as on the GPU."""

    def __init__(self, coefs, omega=0.8, cscale=1.35, fine_presmooth=True, wlevels=(), fine_bf16=False):
        self.omega = omega
        self.cscale = cscale
        self.fine_presmooth = fine_presmooth
        self.wlevels = {int(l) for l in wlevels if int(l) >= 1}
        self.lev = [np.asarray(coefs, f32)]
        while self.lev[-1].shape[1] > 1 or self.lev[-1].shape[3] > 1:
            self.lev.append(coarsen(self.lev[-1]))
        if fine_bf16:  # the finest level's smoother coefficients (and factors) in BF16; coarse grids from FP32
            self.lev[0] = bf16_round(self.lev[0])
        self.fac = [factors(C) for C in self.lev]

    @staticmethod
    def _restrict(res):
        ny, nz, nx = res.shape
        rc = np.zeros(((ny + 1) // 2, nz, (nx + 1) // 2))
        for pj in (0, 1):
            for pi in (0, 1):
                sub = res[pj::2, :, pi::2]
                rc[:sub.shape[0], :, :sub.shape[2]] += sub
        return rc.astype(f32)

    def _level(self, l, r, x):
        """Coarse corrections and post-smoothing of level l < L-1 from iterate x
        (FP32); returns level l's result (FP64 on level 0, FP32 below)."""
        L = len(self.lev)
        w = float(self.omega)
        C = self.lev[l]
        cp, mi = self.fac[l]
        for _ in range(2 if l in self.wlevels else 1):
            rc = self._restrict(np.asarray(r, np.float64) - apply(C, x))
            cpc, mic = self.fac[l + 1]
            if l + 1 == L - 1:
                xc = pre(self.lev[l + 1], cpc, mic, rc, 1.0)        # exact column solve
            else:
                xc = self._level(l + 1, rc, pre(self.lev[l + 1], cpc, mic, rc, w))
            up = np.repeat(np.repeat(xc, 2, axis=0), 2, axis=2)
            ny, nz, nx = x.shape
            x2 = (x + f32(self.cscale) * up[:ny, :, :nx].astype(f32)).astype(f32)
            out = post(C, cp, mi, r, x2, w)
            x = out if l == 0 else out.astype(f32)
        return x

    def __call__(self, r0):
        r0 = np.asarray(r0, np.float64)
        cp, mi = self.fac[0]
        x1 = pre(self.lev[0], cp, mi, r0, float(self.omega)) if self.fine_presmooth else np.zeros(r0.shape, f32)
        if len(self.lev) == 1:
            return x1
        return self._level(0, r0, x1)
