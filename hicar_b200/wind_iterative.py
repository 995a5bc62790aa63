"""Host mirror of HICAR's Fortran module ``wind_iterative``
(src/physics/wind_iterative.F90:39-41): the same public entry points, the same
argument meaning, the same error behaviour, backed by the sm_100a library
through the C ABI of include/hicarw.h.

  init_iter_winds(domain, options)              wind_iterative.F90:215-287
  calc_iter_winds(domain, alpha_in, div_in, adv_den)          :295-532
  finalize_iter_winds()                                       :2142-2267
  probe_lambda_pattern(ca, cb, cc)                            :1096-1115
  probe_zero_corrections(domain)                              :1119-1155
  probe_apply_corrections(domain, adv_den)                    :1158-1163
  probe_record(domain, Tfield, ca, cb, cc, max_leak)          :1169-1231
  probe_finalize(max_leak)                                    :1235-1248

Per-nest state lives in one library handle per nest (the reference's
``domain_cache(MAX_NESTS)``, :139-181); switching nests is O(1).  Where the
reference executes ``stop`` (the solve diverged after every preconditioner
retry, :506-528) this module raises ``SolverDiverged``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

from . import _capi
from .domain import DeviceDomain, mem_kind, ptr

MAX_NESTS = 4  # wind_iterative.F90:139


class SolverDiverged(RuntimeError):
    """The reference stops the model here (wind_iterative.F90:506-528)."""


@dataclasses.dataclass
class WindOptions:
    """The namelist options the solver reads (options%wind, %general, %physics)
    plus this implementation's solve knobs, whose defaults reproduce the reference."""
    wind_solver_iterations: int = 1500      # &wind wind_solver_iterations (namelist_utilities.F90:3871-3876)
    debug: bool = False                     # &general debug
    windtype: int = 1                       # kITERATIVE_WINDS
    advect_density: bool = True             # &adv advect_density
    alpha_const: float = 1.0                # &wind alpha_const
    tol_rel: float = 1.0e-5                 # hard-coded in the reference (:60)
    tol_abs: float = 1.0e-10                # (:59)
    krylov_precision: int = _capi.KRYLOV_F64
    solver: int = _capi.SOLVER_REFERENCE
    criterion: int = _capi.CRIT_RECURRENCE
    replace_every: int = 50
    check_every: int = 8
    precond: int = _capi.PRECOND_JACOBI
    stall_iters: int = 0
    mg_omega: float = 0.8
    fgmres_restart: int = 30
    mg_coarse_scale: float = 1.35          # V-cycle over-correction of the aggregation coarse grid
    mg_skip_fine_presmooth: bool = False   # V-cycle: V(0,1) on the finest level (no pre-smoothing there)
    mg_w_levels: tuple = ()                # levels (>= 1) that correct twice from the coarse grid (W-cycle)
    mg_precision: int = 0                  # 1: BF16 coefficients of the finest level's post-smoother (V(0,1))

    def to_c(self) -> _capi.Options:
        o = _capi.default_options()
        o.max_iters = int(self.wind_solver_iterations)
        o.verbose = int(bool(self.debug) or self.windtype == 1)
        o.tol_rel = float(self.tol_rel)
        o.tol_abs = float(self.tol_abs)
        o.krylov_precision = int(self.krylov_precision)
        o.solver = int(self.solver)
        o.criterion = int(self.criterion)
        o.replace_every = int(self.replace_every)
        o.check_every = int(self.check_every)
        o.precond = int(self.precond)
        o.stall_iters = int(self.stall_iters)
        o.mg_omega = float(self.mg_omega)
        o.fgmres_restart = int(self.fgmres_restart)
        o.mg_coarse_scale = float(self.mg_coarse_scale)
        o.mg_skip_fine_presmooth = int(bool(self.mg_skip_fine_presmooth))
        o.mg_w_levels = sum(1 << int(l) for l in self.mg_w_levels if 1 <= int(l) < 31)
        o.mg_precision = int(self.mg_precision)
        return o


_cache: dict = {}        # nest_indx -> handle
_active: list = [None]   # active nest index
_stream: list = [0]      # CUDA stream handle used for every call (0 = legacy default)


def set_stream(stream_handle: int) -> None:
    _stream[0] = int(stream_handle or 0)


def _handle(nest=None):
    nest = _active[0] if nest is None else nest
    if nest not in _cache:
        raise _capi.HicarwError("wind solver not initialised for this nest: call init_iter_winds first")
    return _cache[nest]


def init_iter_winds(domain: DeviceDomain, options: WindOptions | None = None) -> None:
    """Create (or switch to) the solver state of domain.nest_indx."""
    lib = _capi.load()
    options = options or WindOptions()
    nest = domain.nest_indx
    if nest in _cache:
        _active[0] = nest
        if options is not None:
            _capi.check(lib.hicarw_set_options(_cache[nest], C.byref(options.to_c())), _cache[nest])
        return
    if len(_cache) >= MAX_NESTS:
        raise _capi.HicarwError(f"at most {MAX_NESTS} nests")
    g = _capi.Grid(domain.nx, domain.ny, domain.nz, domain.dx, nest)
    m = _capi.Metrics(*[ptr(domain.metrics[n]) for n in _capi.METRIC_FIELDS])
    h = C.c_void_p()
    kind = mem_kind(domain.metrics["jacobian"])
    rc = lib.hicarw_init_iter_winds(C.byref(g), C.byref(options.to_c()), C.byref(m), kind, _stream[0], C.byref(h))
    _capi.check(rc, None)
    _cache[nest] = h
    _active[0] = nest


def set_options(options: WindOptions, nest=None) -> None:
    h = _handle(nest)
    _capi.check(_capi.load().hicarw_set_options(h, C.byref(options.to_c())), h)


def calc_iter_winds(domain: DeviceDomain, alpha_in, div_in, adv_den: bool) -> dict:
    """Solve for lambda and correct domain.u_dqdt / v_dqdt / w_dqdt in place.
    Returns the solve statistics (status 0/1/2 as the reference's bicgstab_solve)."""
    lib = _capi.load()
    h = _handle(domain.nest_indx)
    st = _capi.Stats()
    kind = mem_kind(domain.u_dqdt)
    rc = lib.hicarw_calc_iter_winds(h, ptr(alpha_in), ptr(div_in), ptr(domain.density) if adv_den else None,
                                    int(bool(adv_den)), ptr(domain.u_dqdt), ptr(domain.v_dqdt), ptr(domain.w_dqdt),
                                    kind, _stream[0], C.byref(st))
    if rc == -4:
        raise SolverDiverged(lib.hicarw_last_error(h).decode())
    _capi.check(rc, h)
    return st.as_dict()


def finalize_iter_winds() -> None:
    lib = _capi.load()
    for nest, h in list(_cache.items()):
        lib.hicarw_finalize_iter_winds(h)
        del _cache[nest]
    _active[0] = None


def probe_lambda_pattern(ca: int, cb: int, cc: int) -> None:
    h = _handle()
    _capi.check(_capi.load().hicarw_probe_lambda_pattern(h, ca, cb, cc, _stream[0]), h)


def probe_zero_corrections(domain: DeviceDomain) -> None:
    h = _handle(domain.nest_indx)
    _capi.check(_capi.load().hicarw_probe_zero_corrections(h, ptr(domain.u_dqdt), ptr(domain.v_dqdt),
                                                            ptr(domain.w_dqdt), mem_kind(domain.u_dqdt),
                                                            _stream[0]), h)


def probe_apply_corrections(domain: DeviceDomain, adv_den: bool) -> None:
    h = _handle(domain.nest_indx)
    _capi.check(_capi.load().hicarw_probe_apply_corrections(
        h, ptr(domain.wind_alpha), ptr(domain.density) if adv_den else None, int(bool(adv_den)),
        ptr(domain.u_dqdt), ptr(domain.v_dqdt), ptr(domain.w_dqdt), mem_kind(domain.u_dqdt), _stream[0]), h)


def probe_record(domain: DeviceDomain, Tfield, ca: int, cb: int, cc: int, max_leak: float) -> float:
    h = _handle(domain.nest_indx)
    ml = C.c_float(max_leak)
    _capi.check(_capi.load().hicarw_probe_record(h, ptr(Tfield), ca, cb, cc, C.byref(ml), mem_kind(Tfield),
                                                 _stream[0]), h)
    return float(ml.value)


def probe_finalize(max_leak: float) -> None:
    h = _handle()
    _capi.check(_capi.load().hicarw_probe_finalize(h, C.c_float(max_leak), _stream[0]), h)


def handle(nest=None):
    """The library handle of a nest (for the extension entry points)."""
    return _handle(nest)
