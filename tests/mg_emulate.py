"""CPU emulation of the multigrid-preconditioned BiCGStab solve, used to choose
the V-cycle's shape: BiCGStab with the GPU schedule's right-preconditioned
recurrences (FP64 vectors), the FP32 V-cycle of mg_ref.VCycle, and the
operator probed by the oracle on a generated case (the oracle's
calibrate_projection_operator, as the first wind update does).  Test
infrastructure, never part of the solver.

    python tests/mg_emulate.py 192 192 40 --alpha smooth --hills 40 --cycles V11,V01,V01-W23

prints the BiCGStab iterations each cycle needs to the relative tolerance.
Cycles: V11 (pre- and post-smoothing on every level, omega 0.8), V01 (no
pre-smoothing on the finest level, omega 1), and V01-W<a><b> (V01 with two
coarse-grid corrections on levels a..b).  The solver's own counts agree: on the
512x512x48 constant-alpha case (seed 1) V11 needs 25 iterations here and on the
GPU."""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import mg_ref  # noqa: E402


def cycle(name: str, coefs, cscale: float = 1.35):
    """mg_ref.VCycle for a cycle name (see the module docstring)."""
    if name == "V11":
        return mg_ref.VCycle(coefs, 0.8, cscale)
    if name == "V01":
        return mg_ref.VCycle(coefs, 1.0, cscale, fine_presmooth=False)
    if name.startswith("V01-W") and len(name) == 7:
        a, b = int(name[5]), int(name[6])
        return mg_ref.VCycle(coefs, 1.0, cscale, fine_presmooth=False, wlevels=range(a, b + 1))
    raise ValueError(f"unknown cycle {name}")


def bicgstab(coefs64, b, M, tol=1e-6, maxit=300):
    """Right-preconditioned BiCGStab (the GPU schedule's recurrences) on the
    interior rows; returns the iterations to ||r|| <= tol ||b|| (-1 if not)."""
    x = np.zeros_like(b)
    r = b.copy()
    rh = r.copy()
    bn = np.linalg.norm(b)
    rho = alpha = om = 1.0
    v = np.zeros_like(b)
    p = np.zeros_like(b)
    for it in range(1, maxit + 1):
        rho1 = np.vdot(rh, r)
        beta = (rho1 / rho) * (alpha / om)
        rho = rho1
        p = r + beta * (p - om * v)
        ph = M(p)
        v = mg_ref.apply(coefs64, ph)
        alpha = rho / np.vdot(rh, v)
        s = r - alpha * v
        sh = M(s)
        t = mg_ref.apply(coefs64, sh)
        om = np.vdot(t, s) / np.vdot(t, t)
        x += alpha * ph + om * sh
        r = s - om * t
        if np.linalg.norm(r) <= tol * bn:
            return it
    return -1


def probed_system(nx, ny, nz, seed=1, alpha="smooth", hills=20):
    """(coefficients (15, ny, nz, nx), right-hand side (ny, nz, nx)) of the
    polishing solve of the first wind update on a generated case."""
    from hicar_b200 import cases
    from oracle import oracle
    case = cases.build_case(nx, ny, nz, seed=seed, adv_den=True, n_hills=hills, alpha=alpha)
    s = oracle.OracleSolver(case.domain)
    fields = lambda: [np.ascontiguousarray(a, dtype=s.dt).copy() for a in (case.u, case.v, case.w)]  # noqa: E731
    u, v, w = fields()
    div = s.divergence(u, v, w, adv_den=True, horz_only=False, use_dqdt=True)
    s.calc_iter_winds(case.alpha, div, case.adv_den, u, v, w)    # analytic solve
    s.calibrate(case.adv_den, u, v, w)                            # probed operator
    u, v, w = fields()
    s.prepare(s.divergence(u, v, w, adv_den=True, horz_only=False, use_dqdt=True))
    return s.coefs(), s.vec("rhs")[1:-1, 1:-1, 1:-1].copy()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("nx", type=int)
    ap.add_argument("ny", type=int)
    ap.add_argument("nz", type=int)
    ap.add_argument("--alpha", default="smooth", choices=["const", "smooth"])
    ap.add_argument("--hills", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--cscale", type=float, default=1.35)
    ap.add_argument("--cycles", default="V11,V01,V01-W23")
    args = ap.parse_args(argv)
    coefs, b = probed_system(args.nx, args.ny, args.nz, args.seed, args.alpha, args.hills)
    c64 = coefs.astype(np.float64)
    out = {}
    for name in args.cycles.split(","):
        t = time.time()
        out[name] = bicgstab(c64, b, cycle(name, coefs, args.cscale), args.tol)
        print(f"{name:8s} iterations {out[name]:4d}  ({time.time() - t:.0f} s)", flush=True)
    return out


if __name__ == "__main__":
    main()
