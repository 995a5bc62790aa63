"""GPU tests of the flexible GMRES(m) outer solver: with the multigrid V-cycle
and with the reference Jacobi-Richardson preconditioner it must reach the
oracle's solution of the same system, its Givens residual estimate must agree
with the FP64 true residual, and restarts must not lose progress."""
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


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def case():
    return cases.build_case(48, 40, 20, seed=4, adv_den=True, n_hills=10)


def _calibrated(case):
    from hicar_b200 import wind, wind_iterative as wi
    from hicar_b200.domain import DeviceDomain
    dom = DeviceDomain.from_case(case, "cuda")
    options = wi.WindOptions()
    wi.init_iter_winds(dom, options)
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    wind.update_winds_iterative(dom, options, div)
    return dom, div


def _coefs(dom):
    from hicar_b200 import wind_iterative as wi
    out = np.empty((15, dom.ny, dom.nz, dom.nx), np.float32)
    h = wi.handle(dom.nest_indx)
    _capi.check(_capi.load().hicarw_get_coefs(h, out.ctypes.data, _capi.MEM_HOST, None), h)
    return out


def _solve(case, dom, div, **kw):
    from hicar_b200 import wind, wind_iterative as wi
    h = wi.handle(dom.nest_indx)
    wi.set_options(wi.WindOptions(tol_rel=1e-9, wind_solver_iterations=3000, **kw))
    dom.set_winds(case.u, case.v, case.w)
    _capi.load().hicarw_reset_solution(h, None)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
    _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
    return st, lam, dom.u_dqdt.cpu().numpy().copy()


@pytest.fixture(scope="module")
def oracle_lambda(oracle_mod, case):
    """The oracle's reference-precision solve of the calibrated system."""
    from hicar_b200 import wind, wind_iterative
    wind_iterative.finalize_iter_winds()
    wind.reset()
    dom, div = _calibrated(case)
    s = oracle_mod.OracleSolver(case.domain)
    s.set_coefs(_coefs(dom), probed=True)
    dom.set_winds(case.u, case.v, case.w)
    wind.calc_divergence(div, dom, use_dqdt=True)
    s.prepare(div.cpu().numpy())
    s.set_vec("x", np.zeros((dom.ny + 2, dom.nz + 2, dom.nx + 2)))
    s.set_tolerance(1e-9)
    st = s.bicgstab(3000)
    assert st["status"] == 0
    lam = s.vec("x").copy()
    wind_iterative.finalize_iter_winds()
    wind.reset()
    return lam


@pytest.mark.parametrize("precond,restart", [(_capi.PRECOND_MG, 30), (_capi.PRECOND_JACOBI, 30),
                                             (_capi.PRECOND_MG, 4)])
def test_fgmres_matches_oracle(case, oracle_lambda, precond, restart):
    dom, div = _calibrated(case)
    st, lam, u = _solve(case, dom, div, solver=_capi.SOLVER_FGMRES, precond=precond, fgmres_restart=restart)
    assert st["status"] == 0
    assert st["precond"] == precond
    # the Givens estimate is a true residual of the FP64 iterate: they agree
    assert st["true_res"] <= 1.05 * st["target"]
    assert st["target"] == pytest.approx(1e-9 * st["b_norm"])
    assert _rel(lam, oracle_lambda) < 1e-5
    # the BiCGStab solution of the same system gives the same winds
    st_b, lam_b, u_b = _solve(case, dom, div, precond=precond, stall_iters=50 if precond else 0)
    assert st_b["status"] == 0
    assert _rel(u, u_b) < 1e-5


def test_fgmres_mg_iterations_and_restart_history(case):
    """MG-preconditioned FGMRES converges in few Arnoldi steps; the recorded
    residual history decreases monotonically across restarts (GMRES minimises
    the residual over each cycle's space and restarts from the updated x)."""
    from hicar_b200 import wind_iterative as wi
    dom, div = _calibrated(case)
    st_j, _, _ = _solve(case, dom, div, solver=_capi.SOLVER_FGMRES, precond=_capi.PRECOND_JACOBI)
    st_m, _, _ = _solve(case, dom, div, solver=_capi.SOLVER_FGMRES, precond=_capi.PRECOND_MG, fgmres_restart=8)
    assert st_m["status"] == 0 and st_j["status"] == 0
    assert st_m["iterations"] * 3 < st_j["iterations"]
    h = wi.handle(dom.nest_indx)
    n = _capi.load().hicarw_get_history(h, None, 0)
    assert n == st_m["iterations"] + 1
    hist = np.empty(n)
    _capi.load().hicarw_get_history(h, hist.ctypes.data, n)
    assert hist[0] == pytest.approx(st_m["res0"])
    assert np.all(hist[1:] <= hist[:-1] * (1 + 1e-6))
