"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/liboracle32.so`` (reference precision: FP32 fields,
FP64 Krylov, as wind_iterative.F90 declares them) or ``liboracle64.so``
(every field in FP64).  Only tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of bench.py use this module, and only as the checker.

Parity status: unpinned by golden vectors (the reference has none for this
path and cannot be compiled here); pinned by the known-answer tests in tests/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

COEF_NAMES = "ABCDEFGHIJKLMNO"
VEC = {"x": 0, "r": 1, "rhat": 2, "p": 3, "phat": 4, "v": 5, "s": 6, "shat": 7, "t": 8,
       "rhs": 9, "Dinv": 10, "pres": 11}


def build() -> None:
    """Compile both oracle builds with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Stats(C.Structure):
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("sweeps", C.c_int), ("retries", C.c_int),
                ("fatal", C.c_int), ("res0", C.c_double), ("res_final", C.c_double),
                ("b_norm", C.c_double), ("target", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_DOM_ARRAYS = ["jacobian", "jacobian_u", "jacobian_v", "jacobian_w", "dzdx", "dzdy", "dzdx_u", "dzdy_v",
               "advection_dz", "neighbor_terrain", "density", "mapfac_mx_u", "mapfac_my_v",
               "mapfac_my_u", "mapfac_mx_v", "mapfac_mxy"]


def _lib(precision: str):
    name = {"ref": "liboracle32.so", "f64": "liboracle64.so"}[precision]
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    vp = C.c_void_p
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [vp, C.c_int]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_calc_iter_winds.restype = C.c_int
    lib.orc_calc_iter_winds.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, vp]
    lib.orc_calc_divergence.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_int, C.c_int]
    lib.orc_calc_updated_winds.argtypes = [vp, C.c_int, vp, vp, vp]
    lib.orc_calc_w_real.argtypes = [vp, vp, vp, vp, vp]
    lib.orc_calc_idealized_wgrid.argtypes = [vp, vp, vp, vp, vp]
    lib.orc_calc_w.argtypes = [vp, vp, vp, C.c_int]
    lib.orc_balance_uvw.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int]
    lib.orc_calc_alpha.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, C.c_int]
    lib.orc_smooth_array.argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int]
    lib.orc_update_stability.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_int, C.c_int, vp, vp]
    lib.orc_spmv.argtypes = [vp, vp, vp]
    lib.orc_apply_precond.argtypes = [vp, vp, vp]
    lib.orc_bicgstab.argtypes = [vp, C.c_int, vp]
    lib.orc_set_tolerance.argtypes = [vp, C.c_double, C.c_double]
    lib.orc_probe_lambda_pattern.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.orc_probe_record.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp]
    lib.orc_probe_finalize.argtypes = [vp]
    lib.orc_calibrate.argtypes = [vp, C.c_int, vp, vp, vp]
    lib.orc_calibrate.restype = C.c_double if precision == "f64" else C.c_float
    lib.orc_build_analytic.argtypes = [vp, vp]
    lib.orc_refresh_coefs.argtypes = [vp, vp]
    lib.orc_prepare_solve.argtypes = [vp, vp]
    lib.orc_set_alpha.argtypes = [vp, vp]
    lib.orc_get_coefs.argtypes = [vp, C.c_int, vp]
    lib.orc_set_coefs.argtypes = [vp, C.c_int, vp]
    lib.orc_set_probed.argtypes = [vp, C.c_int]
    lib.orc_get_vec.argtypes = [vp, C.c_int, vp]
    lib.orc_set_vec.argtypes = [vp, C.c_int, vp]
    lib.orc_set_sweeps.argtypes = [vp, C.c_int]
    lib.orc_set_max_iters.argtypes = [vp, C.c_int]
    lib.orc_get_hist.argtypes = [vp, vp, C.c_int]
    lib.orc_get_hist.restype = C.c_int
    lib.orc_get_stats.argtypes = [vp, vp]
    lib.orc_get_surf.argtypes = [vp, vp, vp, vp]
    lib.orc_true_residual.argtypes = [vp]
    lib.orc_true_residual.restype = C.c_double
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_get_threads.restype = C.c_int
    return lib


_LIBS: dict = {}


def lib(precision: str = "ref"):
    if precision not in _LIBS:
        _LIBS[precision] = _lib(precision)
    return _LIBS[precision]


def set_threads(n: int) -> None:
    for p in ("ref", "f64"):
        lib(p).orc_set_threads(int(n))


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


class OracleSolver:
    """One solver (one nest) of the CPU restatement.

    ``precision='ref'`` keeps the reference's FP32 fields and FP64 Krylov
    vectors; ``'f64'`` runs every field in FP64.  All arrays use the layout of
    ``hicar_b200.cases`` ((ny, nz, nx) C order == Fortran (nx, nz, ny))."""

    def __init__(self, domain, precision: str = "ref", max_iters: int = 1500):
        self.precision = precision
        self.lib = lib(precision)
        self.dt = np.float64 if precision == "f64" else np.float32
        self.d = domain
        self.nx, self.ny, self.nz = domain.nx, domain.ny, domain.nz
        self._keep = {n: np.ascontiguousarray(getattr(domain, n), dtype=self.dt) for n in _DOM_ARRAYS}
        fld = C.c_double if precision == "f64" else C.c_float
        fields = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", fld)] + \
                 [(n, C.c_void_p) for n in _DOM_ARRAYS]
        Dom = type("OrcDomain", (C.Structure,), {"_fields_": fields})
        self._dom = Dom(self.nx, self.ny, self.nz, domain.dx, *[_ptr(self._keep[n]) for n in _DOM_ARRAYS])
        self.h = self.lib.orc_create(C.byref(self._dom), max_iters)
        self.nrows = (self.nx + 2) * (self.ny + 2) * (self.nz + 2)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _a(self, a):
        return np.ascontiguousarray(a, dtype=self.dt)

    # ---- reference entry points ----
    def calc_iter_winds(self, alpha, div, adv_den, u, v, w):
        """calc_iter_winds (wind_iterative.F90:295-532); u, v, w are updated in place
        (they must already have this solver's dtype)."""
        st = Stats()
        for a in (u, v, w):
            assert a.dtype == self.dt and a.flags.c_contiguous
        al, dv = self._a(alpha), self._a(div)
        rc = self.lib.orc_calc_iter_winds(self.h, _ptr(al), _ptr(dv), int(bool(adv_den)), _ptr(u), _ptr(v), _ptr(w),
                                          C.byref(st))
        return rc, st.as_dict()

    def divergence(self, u, v, w, adv_den=True, horz_only=False, use_dqdt=True):
        div = np.empty((self.ny, self.nz, self.nx), self.dt)
        self.lib.orc_calc_divergence(C.byref(self._dom), _ptr(self._a(u)), _ptr(self._a(v)), _ptr(self._a(w)),
                                     _ptr(div), int(bool(adv_den)), int(bool(horz_only)), int(bool(use_dqdt)))
        return div

    def w_real(self, u, v, w_grid=None):
        """calc_w_real (wind.F90:1175-1227) with jaco = jacobian_w."""
        out = np.empty((self.ny, self.nz, self.nx), self.dt)
        self.lib.orc_calc_w_real(C.byref(self._dom), _ptr(self._a(u)), _ptr(self._a(v)),
                                 _ptr(self._a(w_grid)) if w_grid is not None else None, _ptr(out))
        return out

    def idealized_wgrid(self, u, v, w_real_field):
        """calc_idealized_wgrid (wind.F90:940-998): the w_grid predictor."""
        out = np.empty((self.ny, self.nz, self.nx), self.dt)
        self.lib.orc_calc_idealized_wgrid(C.byref(self._dom), _ptr(self._a(u)), _ptr(self._a(v)),
                                          _ptr(self._a(w_real_field)), _ptr(out))
        return out

    def balance_uvw(self, u, v, w, adv_den=True, use_dqdt=True):
        """balance_uvw (wind.F90:123-199): w from the horizontal divergence (w updated in place)."""
        w = self._a(w).copy()
        self.lib.orc_balance_uvw(C.byref(self._dom), _ptr(self._a(u)), _ptr(self._a(v)), _ptr(w),
                                 int(bool(adv_den)), int(bool(use_dqdt)))
        return w

    def calc_alpha(self, froude, halo=1):
        """calc_alpha (wind.F90:1102-1173)."""
        out = np.empty((self.ny, self.nz, self.nx), self.dt)
        self.lib.orc_calc_alpha(self.nx, self.ny, self.nz, _ptr(self._a(froude)), _ptr(out), int(halo))
        return out

    def update_stability(self, u, v, z, theta, froude_terrain=None, froude_mode=True):
        """update_stability (wind.F90:1421-1565): (froude, blk_ri), each (ny, nz, nx);
        froude_terrain has shape (nsect, ny, nz, nx) (Fortran (nx, nz, ny, nsect))."""
        froude = np.empty((self.ny, self.nz, self.nx), self.dt)
        blk_ri = np.empty_like(froude)
        ft = self._a(froude_terrain) if froude_terrain is not None else None
        nsect = int(ft.shape[0]) if ft is not None else 0
        self.lib.orc_update_stability(self.nx, self.ny, self.nz, _ptr(self._a(u)), _ptr(self._a(v)), _ptr(self._a(z)),
                                      _ptr(self._a(theta)), _ptr(ft) if ft is not None else None, nsect,
                                      int(bool(froude_mode)), _ptr(froude), _ptr(blk_ri))
        return froude, blk_ri

    def smooth_array(self, a, window, nsmooths):
        """smooth_array_3d, ydim = 3 (array_utilities.F90:322-397), nsmooths passes."""
        a = self._a(a).copy()
        self.lib.orc_smooth_array(self.nx, self.ny, self.nz, _ptr(a), int(window), int(nsmooths))
        return a

    def updated_winds(self, adv_den, u, v, w):
        self.lib.orc_calc_updated_winds(self.h, int(bool(adv_den)), _ptr(u), _ptr(v), _ptr(w))

    def calibrate(self, adv_den, u, v, w):
        """calibrate_projection_operator (wind.F90:1010-1099); returns the max leakage."""
        return float(self.lib.orc_calibrate(self.h, int(bool(adv_den)), _ptr(u), _ptr(v), _ptr(w)))

    def probe_pattern(self, ca, cb, cc):
        self.lib.orc_probe_lambda_pattern(self.h, ca, cb, cc)

    def probe_record(self, T, ca, cb, cc, max_leak):
        ml = (C.c_double if self.precision == "f64" else C.c_float)(max_leak)
        self.lib.orc_probe_record(self.h, _ptr(self._a(T)), ca, cb, cc, C.byref(ml))
        return float(ml.value)

    def probe_finalize(self):
        self.lib.orc_probe_finalize(self.h)

    # ---- pieces used by the parity tests ----
    def build_analytic(self, alpha):
        self.lib.orc_build_analytic(self.h, _ptr(self._a(alpha)))

    def refresh_coefs(self, alpha):
        self.lib.orc_refresh_coefs(self.h, _ptr(self._a(alpha)))

    def prepare(self, div):
        """extract_diagonal + compute_rhs_3d for this divergence."""
        self.lib.orc_prepare_solve(self.h, _ptr(self._a(div)))

    def set_alpha(self, alpha):
        self.lib.orc_set_alpha(self.h, _ptr(self._a(alpha)))

    def coefs(self) -> np.ndarray:
        out = np.empty((15, self.ny, self.nz, self.nx), self.dt)
        for c in range(15):
            self.lib.orc_get_coefs(self.h, c, _ptr(out[c]))
        return out

    def set_coefs(self, coefs, probed=True):
        for c in range(15):
            self.lib.orc_set_coefs(self.h, c, _ptr(self._a(coefs[c])))
        self.lib.orc_set_probed(self.h, int(bool(probed)))

    def set_probed(self, probed=True):
        self.lib.orc_set_probed(self.h, int(bool(probed)))

    def vec(self, name) -> np.ndarray:
        out = np.empty((self.ny + 2, self.nz + 2, self.nx + 2), np.float64)
        self.lib.orc_get_vec(self.h, VEC[name], _ptr(out))
        return out

    def set_vec(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == (self.ny + 2, self.nz + 2, self.nx + 2)
        self.lib.orc_set_vec(self.h, VEC[name], _ptr(a))

    def spmv(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.lib.orc_spmv(self.h, _ptr(x), _ptr(y))
        return y

    def precond(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.lib.orc_apply_precond(self.h, _ptr(x), _ptr(y))
        return y

    def bicgstab(self, max_iters=None):
        st = Stats()
        self.lib.orc_bicgstab(self.h, int(max_iters or 1500), C.byref(st))
        return st.as_dict()

    def set_tolerance(self, tol_rel, tol_abs=1e-10):
        self.lib.orc_set_tolerance(self.h, tol_rel, tol_abs)

    def set_sweeps(self, n):
        self.lib.orc_set_sweeps(self.h, int(n))

    def set_max_iters(self, n):
        self.lib.orc_set_max_iters(self.h, int(n))

    def history(self) -> np.ndarray:
        n = self.lib.orc_get_hist(self.h, None, 0)
        out = np.empty(max(n, 1), np.float64)
        self.lib.orc_get_hist(self.h, _ptr(out), n)
        return out[:n]

    def stats(self):
        st = Stats()
        self.lib.orc_get_stats(self.h, C.byref(st))
        return st.as_dict()

    def surf(self):
        a = np.empty((self.ny, self.nx), self.dt)
        b = np.empty((self.ny, self.nx), self.dt)
        dzi = np.empty((self.ny, self.nz + 1, self.nx), self.dt)
        self.lib.orc_get_surf(self.h, _ptr(a), _ptr(b), _ptr(dzi))
        return a, b, dzi

    def true_residual(self) -> float:
        return float(self.lib.orc_true_residual(self.h))


def update_winds_first(case, precision="ref", max_iters=1500, tol_rel=None):
    """The first wind update of wind.F90:765-823 at constant alpha: analytic solve,
    calibration by probing, then the polishing solve with the probed operator.
    Returns (solver, u, v, w, stats_first, stats_polish, max_leak)."""
    d = case.domain
    s = OracleSolver(d, precision, max_iters)
    if tol_rel is not None:
        s.set_tolerance(tol_rel)
    dt = s.dt
    u, v, w = (np.ascontiguousarray(a, dtype=dt).copy() for a in (case.u, case.v, case.w))
    div = s.divergence(u, v, w, adv_den=True, horz_only=False, use_dqdt=True)     # wind.F90:805
    rc, st1 = s.calc_iter_winds(case.alpha, div, case.adv_den, u, v, w)            # :807
    leak = s.calibrate(case.adv_den, u, v, w)                                        # :818
    div = s.divergence(u, v, w, adv_den=True, horz_only=False, use_dqdt=True)      # :820
    rc2, st2 = s.calc_iter_winds(case.alpha, div, case.adv_den, u, v, w)           # :821
    return s, u, v, w, st1, st2, leak
