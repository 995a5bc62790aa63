"""GPU tests of the multigrid-preconditioned solve: the V-cycle kernels against
their numpy restatement (tests/mg_ref.py), the preconditioned solve against
the oracle's solution, and the stall detector's fallback to the reference
Jacobi-preconditioned solve."""
import ctypes as C

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


def _calibrated(case, **opt):
    from hicar_b200 import wind, wind_iterative as wi
    from hicar_b200.domain import DeviceDomain
    dom = DeviceDomain.from_case(case, "cuda")
    options = wi.WindOptions(**opt)
    wi.init_iter_winds(dom, options)
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    stats = wind.update_winds_iterative(dom, options, div)
    return dom, options, div, stats


def _coefs(dom):
    from hicar_b200 import wind_iterative as wi
    out = np.empty((15, dom.ny, dom.nz, dom.nx), np.float32)
    h = wi.handle(dom.nest_indx)
    _capi.check(_capi.load().hicarw_get_coefs(h, out.ctypes.data, _capi.MEM_HOST, None), h)
    return out


def test_vcycle_matches_numpy_restatement(case):
    import mg_ref
    from hicar_b200 import wind_iterative as wi
    dom, opt, div, _ = _calibrated(case)
    rng = np.random.default_rng(3)
    x = np.zeros((dom.ny + 2, dom.nz + 2, dom.nx + 2))
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((dom.ny, dom.nz, dom.nx))
    y = np.empty_like(x)
    h = wi.handle(dom.nest_indx)
    _capi.check(_capi.load().hicarw_apply_precond(h, x.ctypes.data, y.ctypes.data, 0, _capi.MEM_HOST, None), h)
    ref = mg_ref.VCycle(_coefs(dom), 0.8)(x[1:-1, 1:-1, 1:-1])
    assert _rel(y[1:-1, 1:-1, 1:-1], ref) < 1e-5
    # boundary rows stay zero
    assert not y[0].any() and not y[:, 0].any() and not y[:, :, 0].any()


def test_mg_solve_matches_oracle_and_cuts_iterations(oracle_mod, case):
    from hicar_b200 import wind, wind_iterative as wi
    dom, opt, div, _ = _calibrated(case)
    u0, v0, w0 = case.u, case.v, case.w  # the divergent input winds, not the corrected ones
    h = wi.handle(dom.nest_indx)
    res = {}
    for name, kw in (("jacobi", {}), ("mg", dict(precond=_capi.PRECOND_MG, stall_iters=50))):
        wi.set_options(wi.WindOptions(tol_rel=1e-9, wind_solver_iterations=3000, **kw))
        dom.set_winds(u0, v0, w0)
        _capi.load().hicarw_reset_solution(h, None)
        wind.calc_divergence(div, dom, use_dqdt=True)
        st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
        lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
        _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
        res[name] = (st, lam, dom.u_dqdt.cpu().numpy().copy())
    st_j, lam_j, u_j = res["jacobi"]
    st_m, lam_m, u_m = res["mg"]
    assert st_j["status"] == 0 and st_m["status"] == 0 and st_m["precond"] == _capi.PRECOND_MG
    assert st_m["iterations"] * 3 < st_j["iterations"]
    assert st_m["true_res"] <= 1.01 * st_m["target"]
    assert st_m["target"] == pytest.approx(1e-9 * st_m["b_norm"])
    # the oracle's reference-precision solve of the same system
    s = oracle_mod.OracleSolver(case.domain)
    s.set_coefs(_coefs(dom), probed=True)
    s.prepare(div.cpu().numpy())
    s.set_vec("x", np.zeros_like(lam_j))
    s.set_tolerance(1e-9)
    st_o = s.bicgstab(3000)
    assert st_o["status"] == 0
    assert _rel(lam_m, s.vec("x")) < 1e-5
    assert _rel(u_m, u_j) < 1e-5


@pytest.mark.parametrize("krylov", [_capi.KRYLOV_F64, _capi.KRYLOV_F32_X64])
def test_stall_falls_back_to_reference_solve(case, krylov):
    """A deliberately useless multigrid damping (omega = 3) makes the
    preconditioned solve stall; the stall detector stops it and the reference
    Jacobi-preconditioned solve, in FP64 Krylov vectors whatever the options
    ask, produces the answer (status 3 = fell back); the next solve runs in the
    options' precision again."""
    from hicar_b200 import wind, wind_iterative as wi
    dom, opt, div, _ = _calibrated(case)
    wi.set_options(wi.WindOptions(tol_rel=1e-6, precond=_capi.PRECOND_MG, stall_iters=10, mg_omega=3.0,
                                  wind_solver_iterations=400, krylov_precision=krylov))
    h = wi.handle(dom.nest_indx)
    _capi.load().hicarw_reset_solution(h, None)
    dom.set_winds(case.u, case.v, case.w)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    assert st["status"] == _capi.HICARW_FELL_BACK
    assert st["precond"] == _capi.PRECOND_JACOBI
    assert st["true_res"] <= 1.01e-6 * st["b_norm"]
    wi.set_options(wi.WindOptions(tol_rel=1e-6, precond=_capi.PRECOND_MG, stall_iters=50,
                                  wind_solver_iterations=400, krylov_precision=krylov))
    _capi.load().hicarw_reset_solution(h, None)
    dom.set_winds(case.u, case.v, case.w)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    assert st["status"] == 0 and st["precond"] == _capi.PRECOND_MG, st
    assert st["true_res"] <= 1.01e-6 * st["b_norm"]


def _fresh_handle(case, monkeypatch, tma):
    """A new handle whose V-cycle is built with the given post-smoother of the
    wide levels: "0" register-fed, "1" tensor copies with the recurrences on
    the consumer warps (post_tma_kernel), "2" tensor copies with the
    recurrences on their own warp (post_tma2_kernel, the default)."""
    from hicar_b200 import wind, wind_iterative as wi
    monkeypatch.setenv("HICARW_MG_TMA", tma)
    wi.finalize_iter_winds()
    wind.reset()
    return _calibrated(case)


@pytest.mark.parametrize("shape", [(131, 75, 21), (128, 96, 16)])
def test_tma_post_smoother_matches_register_path(shape, monkeypatch):
    """Both post-smoothers fed by tensor copies (wide levels: here the finest)
    against the register-fed kernel on the same V-cycle input: bit-identical,
    on a ragged grid (nx not a multiple of the 32-column tile, odd nx and ny,
    nz not a multiple of the 8-level chunk) and a regular one; and against the
    numpy restatement of the V-cycle."""
    import mg_ref
    from hicar_b200 import wind_iterative as wi
    nx, ny, nz = shape
    case = cases.build_case(nx, ny, nz, seed=7, adv_den=True, n_hills=12)
    lib = _capi.load()
    rng = np.random.default_rng(5)
    x = np.zeros((ny + 2, nz + 2, nx + 2))
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((ny, nz, nx))
    out = {}
    for tma in ("0", "1", "2"):
        dom, _, _, _ = _fresh_handle(case, monkeypatch, tma)
        h = wi.handle(dom.nest_indx)
        n0 = lib.hicarw_mg_tma_launches()
        y = np.empty_like(x)
        _capi.check(lib.hicarw_apply_precond(h, x.ctypes.data, y.ctypes.data, 0, _capi.MEM_HOST, None), h)
        out[tma] = (y, lib.hicarw_mg_tma_launches() - n0, _coefs(dom))
    assert out["0"][1] == 0 and out["1"][1] >= 1 and out["2"][1] >= 1
    for tma in ("1", "2"):
        np.testing.assert_array_equal(out[tma][2], out["0"][2])
        np.testing.assert_array_equal(out[tma][0], out["0"][0])
    ref = mg_ref.VCycle(out["2"][2], 0.8)(x[1:-1, 1:-1, 1:-1])
    assert _rel(out["2"][0][1:-1, 1:-1, 1:-1], ref) < 1e-5
    y = out["2"][0]
    assert not y[0].any() and not y[-1].any() and not y[:, 0].any() and not y[:, -1].any()
    assert not y[:, :, 0].any() and not y[:, :, -1].any()


@pytest.mark.parametrize("shape", [(131, 75, 21), (128, 96, 16), (161, 131, 21)])
def test_tma_post_smoother_zero_iterate_matches_register_path(shape, monkeypatch):
    """V(0,1) on the finest level (its iterate zero, x2 = s P xc read straight
    from the staged coarse rows): the tensor-copy post-smoother against the
    register-fed kernel, bit-identical, on ragged grids (odd nx and ny, so the
    last aggregate of a row has one column; nz not a multiple of the 8-level
    chunk) and a regular one; on 161 x 131 level 1 (81 x 66 columns) takes
    the wide restriction tiles."""
    from hicar_b200 import wind_iterative as wi
    nx, ny, nz = shape
    case = cases.build_case(nx, ny, nz, seed=17, adv_den=True, n_hills=12)
    lib = _capi.load()
    rng = np.random.default_rng(23)
    x = np.zeros((ny + 2, nz + 2, nx + 2))
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((ny, nz, nx))
    out = {}
    for tma in ("0", "2"):
        dom, _, _, _ = _fresh_handle(case, monkeypatch, tma)
        h = wi.handle(dom.nest_indx)
        wi.set_options(wi.WindOptions(mg_skip_fine_presmooth=True, mg_omega=1.0, mg_coarse_scale=1.35))
        n0 = lib.hicarw_mg_tma_launches()
        y = np.empty_like(x)
        _capi.check(lib.hicarw_apply_precond(h, x.ctypes.data, y.ctypes.data, 0, _capi.MEM_HOST, None), h)
        out[tma] = (y, lib.hicarw_mg_tma_launches() - n0)
    assert out["0"][1] == 0 and out["2"][1] >= 1
    np.testing.assert_array_equal(out["2"][0], out["0"][0])
    y = out["2"][0]
    assert not y[0].any() and not y[-1].any() and not y[:, 0].any() and not y[:, -1].any()
    assert not y[:, :, 0].any() and not y[:, :, -1].any()


def test_tma_post_smoother_solve_identical(monkeypatch):
    """A whole multigrid-preconditioned solve (BiCGStab, CUDA graphs of
    iterations) with and without the tensor-copy post-smoother: the same
    iteration count and the same lambda, bit for bit."""
    from hicar_b200 import wind, wind_iterative as wi
    case = cases.build_case(131, 75, 21, seed=8, adv_den=True, n_hills=12)
    lib = _capi.load()
    res = {}
    for tma in ("0", "1", "2"):
        dom, _, div, _ = _fresh_handle(case, monkeypatch, tma)
        h = wi.handle(dom.nest_indx)
        wi.set_options(wi.WindOptions(tol_rel=1e-8, precond=_capi.PRECOND_MG, stall_iters=50))
        n0 = lib.hicarw_mg_tma_launches()
        dom.set_winds(case.u, case.v, case.w)
        lib.hicarw_reset_solution(h, None)
        wind.calc_divergence(div, dom, use_dqdt=True)
        st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
        lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
        _capi.check(lib.hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None), h)
        res[tma] = (st, lam, lib.hicarw_mg_tma_launches() - n0)
    assert res["0"][2] == 0 and res["1"][2] >= 1 and res["2"][2] >= 1
    for tma in ("0", "1", "2"):
        assert res[tma][0]["status"] == 0 and res[tma][0]["precond"] == _capi.PRECOND_MG
    for tma in ("1", "2"):
        assert res[tma][0]["iterations"] == res["0"][0]["iterations"]
        np.testing.assert_array_equal(res[tma][1], res["0"][1])
