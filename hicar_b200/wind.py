"""Host mirror of the solver-facing part of HICAR's ``wind.F90``:
``calc_divergence`` (wind.F90:250-523), ``calibrate_projection_operator``
(:1010-1099) and the iterative-winds branch of ``update_winds`` (:765-823).
All arithmetic runs in the CUDA library; this module only orders the calls.
"""
from __future__ import annotations

import ctypes as C

from . import _capi
from . import wind_iterative as wi
from .domain import DeviceDomain, mem_kind, ptr

_operator_calibrated: dict = {}  # per nest (wind.F90 operator_calibrated)


def calc_divergence(div, domain: DeviceDomain, advect_density: bool = True, horz_only: bool = False,
                    use_dqdt: bool = False) -> None:
    """div = D(u, v, w) (wind.F90:250-523).  use_dqdt selects the dqdt winds."""
    h = wi.handle(domain.nest_indx)
    u, v, w = (domain.u_dqdt, domain.v_dqdt, domain.w_dqdt) if use_dqdt else (domain.u, domain.v, domain.w)
    if u is None:
        raise ValueError("data_3d winds are not set on this domain (use_dqdt=False)")
    rc = _capi.load().hicarw_calc_divergence(h, ptr(u), ptr(v), ptr(w), ptr(domain.density) if advect_density else None,
                                             ptr(div), int(bool(advect_density)), int(bool(horz_only)),
                                             int(bool(use_dqdt)), mem_kind(u), wi._stream[0])
    _capi.check(rc, h)


def calibrate_projection_operator(domain: DeviceDomain, options: wi.WindOptions, div=None,
                                  on_device: bool = True) -> float:
    """Calibrate A = 2 D o G by the 27-colouring probe (wind.F90:1010-1099).

    on_device=True runs all 27 probes inside the library (no host round trip);
    on_device=False drives the reference's probe hooks one by one, exactly as
    wind.F90:1055-1067 does (``div`` is the probe's scratch divergence)."""
    lib = _capi.load()
    h = wi.handle(domain.nest_indx)
    adv = bool(options.advect_density)
    if on_device:
        leak = C.c_float(0.0)
        rc = lib.hicarw_calibrate_projection_operator(h, ptr(domain.wind_alpha), ptr(domain.density) if adv else None,
                                                      int(adv), ptr(domain.u_dqdt), ptr(domain.v_dqdt),
                                                      ptr(domain.w_dqdt), C.byref(leak), mem_kind(domain.u_dqdt),
                                                      wi._stream[0])
        _capi.check(rc, h)
        return float(leak.value)
    saved = [a.clone() if hasattr(a, "clone") else a.copy() for a in (domain.u_dqdt, domain.v_dqdt, domain.w_dqdt)]
    max_leak = 0.0
    for cc in range(3):
        for cb in range(3):
            for ca in range(3):
                wi.probe_lambda_pattern(ca, cb, cc)
                wi.probe_zero_corrections(domain)
                wi.probe_apply_corrections(domain, adv)
                calc_divergence(div, domain, advect_density=adv, horz_only=False, use_dqdt=True)
                max_leak = wi.probe_record(domain, div, ca, cb, cc, max_leak)
    wi.probe_finalize(max_leak)
    domain.set_winds(*saved)
    return max_leak


def update_winds_iterative(domain: DeviceDomain, options: wi.WindOptions, div) -> list:
    """The iterative-winds branch of update_winds (wind.F90:765-823) for a
    constant alpha already stored in domain.wind_alpha: first update = analytic
    solve, calibration, polishing solve; later updates = one solve."""
    nest = domain.nest_indx
    stats = []
    calc_divergence(div, domain, horz_only=False, use_dqdt=True)                              # :805
    stats.append(wi.calc_iter_winds(domain, domain.wind_alpha, div, options.advect_density))  # :807
    if not _operator_calibrated.get(nest, False):                                             # :813
        calibrate_projection_operator(domain, options, div)                                   # :814
        _operator_calibrated[nest] = True
        calc_divergence(div, domain, horz_only=False, use_dqdt=True)                          # :817
        stats.append(wi.calc_iter_winds(domain, domain.wind_alpha, div, options.advect_density))
    return stats


def reset() -> None:
    _operator_calibrated.clear()


# ---- the steps either side of the solve (device arrays) ----------------------
def _s():
    return wi._stream[0]


def calc_w_real(domain: DeviceDomain, u, v, w_grid, w_real) -> None:
    """calc_w_real (wind.F90:1175-1227) with jaco = jacobian_w; w_grid None = zero."""
    h = wi.handle(domain.nest_indx)
    _capi.check(_capi.load().hicarw_calc_w_real(h, ptr(u), ptr(v), ptr(w_grid) if w_grid is not None else None,
                                                ptr(w_real), _capi.MEM_DEVICE, _s()), h)


def calc_idealized_wgrid(domain: DeviceDomain, w_real) -> None:
    """calc_idealized_wgrid (wind.F90:940-998): domain.w_dqdt from the dqdt winds and w_real."""
    h = wi.handle(domain.nest_indx)
    _capi.check(_capi.load().hicarw_calc_idealized_wgrid(h, ptr(domain.u_dqdt), ptr(domain.v_dqdt), ptr(w_real),
                                                         ptr(domain.w_dqdt), _capi.MEM_DEVICE, _s()), h)


def balance_uvw(domain: DeviceDomain, adv_den: bool, update: bool = False) -> None:
    """balance_uvw (wind.F90:123-199): w (dqdt winds if update, else data winds)
    from the horizontal divergence of u and v."""
    h = wi.handle(domain.nest_indx)
    u, v, w = (domain.u_dqdt, domain.v_dqdt, domain.w_dqdt) if update else (domain.u, domain.v, domain.w)
    _capi.check(_capi.load().hicarw_balance_uvw(h, ptr(u), ptr(v), ptr(domain.density), ptr(w), int(bool(adv_den)),
                                                int(bool(update)), _capi.MEM_DEVICE, _s()), h)


def update_stability(domain: DeviceDomain, z, theta, froude, blk_ri, froude_terrain=None,
                     froude_mode: bool = True) -> None:
    """update_stability (wind.F90:1421-1565): blk_ri and (froude_mode: alpha_const < 0
    with iterative winds) the Froude number from the dqdt winds, the mass-level
    heights z, the potential temperature theta and the sector blocking heights
    froude_terrain (nsect, ny, nz, nx)."""
    h = wi.handle(domain.nest_indx)
    nsect = int(froude_terrain.shape[0]) if froude_terrain is not None else 0
    _capi.check(_capi.load().hicarw_update_stability(
        h, ptr(domain.u_dqdt), ptr(domain.v_dqdt), ptr(z), ptr(theta),
        ptr(froude_terrain) if froude_terrain is not None else None, nsect, int(bool(froude_mode)), ptr(froude),
        ptr(blk_ri), _capi.MEM_DEVICE, _s()), h)


def calc_alpha(domain: DeviceDomain, froude, halo: int = 1, window: int = 2, nsmooths: int = 3) -> None:
    """calc_alpha (wind.F90:1102-1173) into domain.wind_alpha, then the smoothing of
    update_winds (:784: windowsize 2, clamped to the halo width, 3 passes)."""
    h = wi.handle(domain.nest_indx)
    lib = _capi.load()
    _capi.check(lib.hicarw_calc_alpha(h, ptr(froude), ptr(domain.wind_alpha), int(halo), _capi.MEM_DEVICE, _s()), h)
    _capi.check(lib.hicarw_smooth_alpha(h, ptr(domain.wind_alpha), min(int(window), int(halo)), int(nsmooths),
                                        _capi.MEM_DEVICE, _s()), h)
