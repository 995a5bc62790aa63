"""CPU checks of the C ABI library: it loads, exports every entry point that
include/hicarw.h declares, and its default options are the reference's
constants (no compute call: there is no GPU here)."""
import ctypes as C
import os
import re

from hicar_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "hicarw.h")).read()
    return sorted(set(re.findall(r"\b(hicarw_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_capi.EXPORTS) == names


def test_default_options_are_reference_constants(lib):
    o = _capi.default_options()
    assert o.max_iters == 1500            # namelist_utilities.F90:3871-3876
    assert o.tol_rel == 1.0e-5            # wind_iterative.F90:60
    assert o.tol_abs == 1.0e-10           # wind_iterative.F90:59
    assert o.krylov_precision == _capi.KRYLOV_F64
    assert o.solver == _capi.SOLVER_REFERENCE


def test_options_mirror_matches_the_c_struct(lib):
    """The ctypes mirror of hicarw_options has the C struct's size and field
    order: the library's defaults land in the expected fields and nothing is
    written past the mirror's end."""
    n = C.sizeof(_capi.Options)
    buf = (C.c_ubyte * (n + 64))(*([0xA5] * (n + 64)))
    lib.hicarw_default_options(C.cast(buf, C.POINTER(_capi.Options)))
    assert bytes(buf[n:]) == b"\xa5" * 64
    o = _capi.Options.from_buffer_copy(bytes(buf[:n]))
    assert o.check_every == 8 and o.replace_every == 50 and o.precond == _capi.PRECOND_JACOBI
    assert o.stall_iters == 0 and o.fgmres_restart == 30
    assert abs(o.mg_omega - 0.8) < 1e-7 and abs(o.mg_coarse_scale - 1.35) < 1e-7
    assert o.mg_skip_fine_presmooth == 0
    from hicar_b200 import wind_iterative as wi
    c = wi.WindOptions(mg_skip_fine_presmooth=True, mg_omega=1.0).to_c()
    assert c.mg_skip_fine_presmooth == 1 and c.mg_omega == 1.0


def test_bad_arguments_are_errors_not_aborts(lib):
    h = C.c_void_p()
    g = _capi.Grid(1, 1, 1, 250.0, 1)     # too small: rejected before any CUDA call
    rc = lib.hicarw_init_iter_winds(C.byref(g), None, None, 0, None, C.byref(h))
    assert rc == -1
    assert lib.hicarw_finalize_iter_winds(None) == -1
    assert lib.hicarw_calc_iter_winds(None, None, None, None, 0, None, None, None, 0, None, None) == -1


def test_unknown_krylov_precision_is_rejected_before_cuda(lib):
    """An out-of-range krylov_precision is an argument error, returned before
    any CUDA call (valid grid and metrics otherwise)."""
    h = C.c_void_p()
    g = _capi.Grid(16, 16, 8, 250.0, 1)
    m = _capi.Metrics()
    o = _capi.default_options()
    for bad in (-1, 3, 99):
        o.krylov_precision = bad
        assert lib.hicarw_init_iter_winds(C.byref(g), C.byref(o), C.byref(m), 0, None, C.byref(h)) == -1
        assert not h.value
