"""GPU tests of two pieces of the host contract that no solve exercises on its
own:

* Nest switching.  HICAR keeps one solver state per nest and switches between
  them on a nest change (wind_iterative.F90:2613-2851, save_to_cache /
  restore_from_cache, up to MAX_NESTS = 4).  Here every nest owns a library
  handle, so a switch copies nothing; two nests of different sizes solved
  alternately must each give the same lambda and winds, bit for bit, as the
  same nest solved alone.
* Bounded device waits.  Every mbarrier wait of the tensor-copy smoother and
  the tensor-core convolutions gives up after a limit, records an error flag
  and returns.  hicarw_debug_wait_timeout runs that wait on a barrier nothing
  completes, with a limit of a few microseconds: the call must report
  HICARW_ERR_TIMEOUT, and a solve on the same handle right after must succeed
  and match a solve on a fresh handle.

Collected after the other solver tests (the allocation-free entry point's
file comes last)."""
import numpy as np
import pytest

from hicar_b200 import _capi, cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _fresh(lib):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hicar_b200 import wind, wind_iterative
    wind_iterative.finalize_iter_winds()
    wind.reset()
    yield
    wind_iterative.finalize_iter_winds()
    wind.reset()


OPT = dict(tol_rel=1e-8, wind_solver_iterations=3000, precond=_capi.PRECOND_MG, stall_iters=50)


def _domain(case, nest):
    from hicar_b200.domain import DeviceDomain
    return DeviceDomain.from_case(case, "cuda", nest_indx=nest)


def _first_update(dom, opt):
    from hicar_b200 import wind, wind_iterative as wi
    wi.init_iter_winds(dom, opt)
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    wind.update_winds_iterative(dom, opt, div)
    return div


def _solve(dom, div, case):
    from hicar_b200 import wind, wind_iterative as wi
    wi.init_iter_winds(dom, None)  # switch to this nest (no copy)
    wi.set_options(wi.WindOptions(**OPT), nest=dom.nest_indx)
    h = wi.handle(dom.nest_indx)
    dom.set_winds(case.u, case.v, case.w)
    _capi.load().hicarw_reset_solution(h, None)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
    _capi.check(_capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None), h)
    return st, lam, [a.cpu().numpy().copy() for a in (dom.u_dqdt, dom.v_dqdt, dom.w_dqdt)]


def test_nest_switching_matches_single_nest_solves():
    from hicar_b200 import wind, wind_iterative as wi
    ca = cases.build_case(48, 40, 16, seed=41, adv_den=True, n_hills=6)
    cb = cases.build_case(36, 44, 12, seed=43, adv_den=True, n_hills=5, alpha="smooth")
    alone = {}
    for nest, case in ((1, ca), (2, cb)):
        dom = _domain(case, nest)
        div = _first_update(dom, wi.WindOptions())
        alone[nest] = _solve(dom, div, case)
        wi.finalize_iter_winds()
        wind.reset()
    doms = {1: _domain(ca, 1), 2: _domain(cb, 2)}
    divs = {n: _first_update(doms[n], wi.WindOptions()) for n in (1, 2)}
    assert len(wi._cache) == 2
    for rep in range(2):
        for nest, case in ((1, ca), (2, cb)):
            st, lam, winds = _solve(doms[nest], divs[nest], case)
            st0, lam0, winds0 = alone[nest]
            assert st["status"] == 0 and st["iterations"] == st0["iterations"], (nest, rep)
            np.testing.assert_array_equal(lam, lam0)
            for g, r in zip(winds, winds0):
                np.testing.assert_array_equal(g, r)


def test_bounded_wait_times_out_and_handle_stays_usable():
    from hicar_b200 import wind, wind_iterative as wi
    case = cases.build_case(128, 80, 20, seed=47, adv_den=True, n_hills=6)  # wide enough for the tensor-copy smoother
    dom = _domain(case, 1)
    div = _first_update(dom, wi.WindOptions())
    st0, lam0, winds0 = _solve(dom, div, case)
    h = wi.handle(1)
    lib = _capi.load()
    assert lib.hicarw_debug_wait_timeout(h, 5.0, None) == -6  # HICARW_ERR_TIMEOUT
    assert b"timed out" in lib.hicarw_last_error(h)
    assert lib.hicarw_debug_wait_timeout(h, 0.0, None) == -1  # limit outside 1 .. 1e5 us
    st, lam, winds = _solve(dom, div, case)
    assert st["status"] == 0 and st["iterations"] == st0["iterations"]
    np.testing.assert_array_equal(lam, lam0)
    for g, r in zip(winds, winds0):
        np.testing.assert_array_equal(g, r)
    assert _capi.load().hicarw_mg_tma_launches() > 0
