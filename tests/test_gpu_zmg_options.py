"""GPU tests of the solver options beyond the default configuration: V(0,1)
on the finest level, W-cycles on chosen coarse levels, FP32 Krylov vectors with
FP64 lambda, and the opt-in column-marching operator kernels.  Kept in a file
that pytest collects after the tests of the default configuration (and before
the allocation-free entry point's), so that a failure of an option cannot stop
a `-x` run before those have run."""
import os

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


@pytest.mark.parametrize("shape", [(48, 40, 20), (197, 101, 13)])
def test_vcycle_without_fine_presmoothing(shape):
    """V(0,1) on the finest level (mg_skip_fine_presmooth): level 1 restricts
    the input itself and the finest post-smoother starts from the coarse
    correction alone; against the numpy restatement, on a grid whose levels 0
    and 1 use the small-level tiles and on a ragged one whose level 0 uses the
    tensor-copy post-smoother and level 1 the wide restriction tiles
    (99 x 51 coarse columns, nz not a multiple of 8)."""
    import mg_ref
    from hicar_b200 import wind_iterative as wi
    nx, ny, nz = shape
    case = cases.build_case(nx, ny, nz, seed=9, adv_den=True, n_hills=10)
    dom, _, _, _ = _calibrated(case)
    h = wi.handle(dom.nest_indx)
    lib = _capi.load()
    rng = np.random.default_rng(11)
    x = np.zeros((ny + 2, nz + 2, nx + 2))
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((ny, nz, nx))
    coefs = _coefs(dom)
    for skip, omega in ((False, 0.8), (True, 1.0), (False, 0.8)):  # switching the option back and forth
        wi.set_options(wi.WindOptions(mg_skip_fine_presmooth=skip, mg_omega=omega))
        y = np.empty_like(x)
        _capi.check(lib.hicarw_apply_precond(h, x.ctypes.data, y.ctypes.data, 0, _capi.MEM_HOST, None), h)
        ref = mg_ref.VCycle(coefs, omega, fine_presmooth=not skip)(x[1:-1, 1:-1, 1:-1])
        assert _rel(y[1:-1, 1:-1, 1:-1], ref) < 1e-5, (skip, omega)
        assert not y[0].any() and not y[:, 0].any() and not y[:, :, 0].any()


def test_mg_solve_without_fine_presmoothing(oracle_mod, case):
    """The multigrid-preconditioned solve with V(0,1) on the finest level
    (omega = 1) converges to the same lambda as the oracle's reference solve."""
    from hicar_b200 import wind, wind_iterative as wi
    dom, opt, div, _ = _calibrated(case)
    h = wi.handle(dom.nest_indx)
    wi.set_options(wi.WindOptions(tol_rel=1e-9, wind_solver_iterations=3000, precond=_capi.PRECOND_MG,
                                  stall_iters=50, mg_skip_fine_presmooth=True, mg_omega=1.0))
    dom.set_winds(case.u, case.v, case.w)
    _capi.load().hicarw_reset_solution(h, None)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    assert st["status"] == 0 and st["precond"] == _capi.PRECOND_MG
    assert st["true_res"] <= 1.01 * st["target"]
    lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
    _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
    s = oracle_mod.OracleSolver(case.domain)
    s.set_coefs(_coefs(dom), probed=True)
    s.prepare(div.cpu().numpy())
    s.set_vec("x", np.zeros_like(lam))
    s.set_tolerance(1e-9)
    assert s.bicgstab(3000)["status"] == 0
    assert _rel(lam, s.vec("x")) < 1e-5


@pytest.mark.parametrize("shape,wlev", [((48, 40, 20), (1, 2)), ((197, 101, 13), (2, 3))])
def test_vcycle_w_levels(shape, wlev):
    """W-cycle on chosen coarse levels (mg_w_levels; with V(0,1) on the finest
    level and omega = 1) against the numpy restatement, then back to the plain
    V-cycle on the same handle."""
    import mg_ref
    from hicar_b200 import wind_iterative as wi
    nx, ny, nz = shape
    case = cases.build_case(nx, ny, nz, seed=13, adv_den=True, n_hills=10)
    dom, _, _, _ = _calibrated(case)
    h = wi.handle(dom.nest_indx)
    lib = _capi.load()
    rng = np.random.default_rng(17)
    x = np.zeros((ny + 2, nz + 2, nx + 2))
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((ny, nz, nx))
    coefs = _coefs(dom)
    for opt, ref in ((dict(mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=wlev),
                      dict(omega=1.0, fine_presmooth=False, wlevels=wlev)),
                     (dict(), dict(omega=0.8))):
        wi.set_options(wi.WindOptions(**opt))
        y = np.empty_like(x)
        _capi.check(lib.hicarw_apply_precond(h, x.ctypes.data, y.ctypes.data, 0, _capi.MEM_HOST, None), h)
        want = mg_ref.VCycle(coefs, **ref)(x[1:-1, 1:-1, 1:-1])
        assert _rel(y[1:-1, 1:-1, 1:-1], want) < 1e-5, opt
        assert not y[0].any() and not y[:, 0].any() and not y[:, :, 0].any()


def test_mg_solve_w_levels(oracle_mod, case):
    """The multigrid-preconditioned solve with a W-cycle on levels 1-2 (V(0,1)
    on the finest level, omega = 1) converges to the oracle's lambda."""
    from hicar_b200 import wind, wind_iterative as wi
    dom, opt, div, _ = _calibrated(case)
    h = wi.handle(dom.nest_indx)
    wi.set_options(wi.WindOptions(tol_rel=1e-9, wind_solver_iterations=3000, precond=_capi.PRECOND_MG,
                                  stall_iters=50, mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=(1, 2)))
    dom.set_winds(case.u, case.v, case.w)
    _capi.load().hicarw_reset_solution(h, None)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    assert st["status"] == 0 and st["precond"] == _capi.PRECOND_MG
    assert st["true_res"] <= 1.01 * st["target"]
    lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
    _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
    s = oracle_mod.OracleSolver(case.domain)
    s.set_coefs(_coefs(dom), probed=True)
    s.prepare(div.cpu().numpy())
    s.set_vec("x", np.zeros_like(lam))
    s.set_tolerance(1e-9)
    assert s.bicgstab(3000)["status"] == 0
    assert _rel(lam, s.vec("x")) < 1e-5


@pytest.mark.parametrize("shape", [(48, 40, 20), (197, 101, 13), (132, 37, 9), (8, 6, 5)])
def test_column_marching_operator_matches_row_kernels(shape, monkeypatch):
    """The column-marching operator applies (HICARW_SPMV_MARCH=1: scalar, one
    column per lane; unset: four columns per lane with 16-byte loads where nx
    is a multiple of 4) give the row kernels' FP64 values bit for bit, identity
    rows included: on a grid narrower than one strip in places, a ragged one
    (nx odd: the row kernels serve the float4 setting), one whose last strip
    holds a single lane, and one of two float4 groups."""
    from hicar_b200 import wind_iterative as wi
    nx, ny, nz = shape
    case = cases.build_case(nx, ny, nz, seed=19, adv_den=True, n_hills=10)
    dom, _, _, _ = _calibrated(case)
    h = wi.handle(dom.nest_indx)
    lib = _capi.load()
    x = np.random.default_rng(23).standard_normal((ny + 2, nz + 2, nx + 2))
    out = {}
    for march in ("0", "1", "4"):
        if march == "4":
            monkeypatch.delenv("HICARW_SPMV_MARCH", raising=False)
        else:
            monkeypatch.setenv("HICARW_SPMV_MARCH", march)
        y = np.empty_like(x)
        _capi.check(lib.hicarw_apply_operator(h, x.ctypes.data, y.ctypes.data, _capi.MEM_HOST, None), h)
        out[march] = y
    np.testing.assert_array_equal(out["1"], out["0"])
    np.testing.assert_array_equal(out["4"], out["0"])


@pytest.mark.parametrize("prec", [_capi.KRYLOV_F64, _capi.KRYLOV_F32_X64])
def test_column_marching_solve(case, monkeypatch, prec):
    """The multigrid-preconditioned solve with the column-marching sigma and
    five-dot kernels (scalar and float4), FP64 and FP32 Krylov vectors: the
    same lambda as with the row kernels (the reductions sum in another order,
    so to the solve tolerance), iterations within one."""
    from hicar_b200 import wind, wind_iterative as wi
    res = {}
    for march in ("0", "1", "4"):
        if march == "4":
            monkeypatch.delenv("HICARW_SPMV_MARCH", raising=False)
        else:
            monkeypatch.setenv("HICARW_SPMV_MARCH", march)
        wi.finalize_iter_winds()
        wind.reset()
        dom, _, div, _ = _calibrated(case)
        h = wi.handle(dom.nest_indx)
        wi.set_options(wi.WindOptions(tol_rel=1e-9, wind_solver_iterations=3000, precond=_capi.PRECOND_MG,
                                      stall_iters=50, krylov_precision=prec))
        dom.set_winds(case.u, case.v, case.w)
        _capi.load().hicarw_reset_solution(h, None)
        wind.calc_divergence(div, dom, use_dqdt=True)
        st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
        lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
        _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
        res[march] = (st, lam)
    for march in ("1", "4"):
        assert res[march][0]["status"] == 0
        assert abs(res[march][0]["iterations"] - res["0"][0]["iterations"]) <= 1
        assert _rel(res[march][1], res["0"][1]) < 1e-6


@pytest.mark.parametrize("wlev", [(), (1, 2)])
def test_mg_solve_fp32_vectors_fp64_lambda(case, wlev):
    """FP32 Krylov vectors with FP64 reductions and FP64 accumulation of lambda
    (HICARW_KRYLOV_F32_X64), multigrid-preconditioned, at the benchmark's 1e-6:
    the FP64 true residual meets the tolerance, and the iterations, lambda and
    winds follow the FP64-vector solve of the same system."""
    from hicar_b200 import wind, wind_iterative as wi
    dom, _, div, _ = _calibrated(case)
    h = wi.handle(dom.nest_indx)
    cyc = dict(mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=wlev) if wlev else {}
    res = {}
    for prec in (_capi.KRYLOV_F64, _capi.KRYLOV_F32_X64):
        wi.set_options(wi.WindOptions(tol_rel=1e-6, wind_solver_iterations=3000, precond=_capi.PRECOND_MG,
                                      stall_iters=50, krylov_precision=prec, **cyc))
        dom.set_winds(case.u, case.v, case.w)
        _capi.load().hicarw_reset_solution(h, None)
        wind.calc_divergence(div, dom, use_dqdt=True)
        st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
        lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
        _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
        res[prec] = (st, lam, dom.u_dqdt.cpu().numpy().copy())
    st64, lam64, u64 = res[_capi.KRYLOV_F64]
    st32, lam32, u32 = res[_capi.KRYLOV_F32_X64]
    assert st32["status"] == 0 and st32["precond"] == _capi.PRECOND_MG
    assert 0.0 <= st32["true_res"] <= 1.01 * st32["target"]
    assert abs(st32["iterations"] - st64["iterations"]) <= 2
    assert _rel(lam32, lam64) < 1e-5
    assert _rel(u32, u64) < 1e-5


def _profile_names(h):
    """Kernel names of one profiled solve iteration of the handle's configuration."""
    import ctypes as C
    lib = _capi.load()
    cap = 64
    names = C.create_string_buffer(32 * cap)
    ms, by = (C.c_double * cap)(), (C.c_double * cap)()
    cnt = (C.c_int * cap)()
    n = lib.hicarw_profile_iteration(h, 1, names, ms, by, cnt, cap, None)
    assert n > 0
    return [names.raw[32 * q:32 * q + 32].split(b"\0")[0].decode() for q in range(n)]


@pytest.mark.parametrize("shape", [(48, 40, 20), (197, 101, 13), (130, 66, 24)])
def test_fused_coarse_cycle_bitexact(shape, monkeypatch):
    """The coarse part of the cycle run by one thread-block cluster (levels of
    at most 256 columns; the default) gives the per-level launches' V-cycle bit
    for bit, for the V-cycle and for W-cycles that reach into the fused levels,
    on a small grid, a ragged one and one with odd coarse extents."""
    from hicar_b200 import wind, wind_iterative as wi
    nx, ny, nz = shape
    case = cases.build_case(nx, ny, nz, seed=21, adv_den=True, n_hills=8)
    rng = np.random.default_rng(29)
    x = np.zeros((ny + 2, nz + 2, nx + 2))
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((ny, nz, nx))
    cycles = [dict(), dict(mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=(2, 3)),
              dict(mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=(2, 3, 4, 5))]
    out = {}
    for fuse in ("0", "1"):
        monkeypatch.setenv("HICARW_MG_FUSE", fuse)
        wi.finalize_iter_winds()
        wind.reset()
        dom, _, _, _ = _calibrated(case, precond=_capi.PRECOND_MG, stall_iters=50)
        h = wi.handle(dom.nest_indx)
        lib = _capi.load()
        for q, cyc in enumerate(cycles):
            wi.set_options(wi.WindOptions(precond=_capi.PRECOND_MG, stall_iters=50, **cyc))
            y = np.empty_like(x)
            _capi.check(lib.hicarw_apply_precond(h, x.ctypes.data, y.ctypes.data, 0, _capi.MEM_HOST, None), h)
            out[(fuse, q)] = y
            fused = any(n.startswith("mg_coarse_l") for n in _profile_names(h))
            assert fused == (fuse == "1"), (fuse, q)
    for q in range(len(cycles)):
        np.testing.assert_array_equal(out[("1", q)], out[("0", q)])


def test_fused_coarse_cycle_solve(case, monkeypatch):
    """A multigrid-preconditioned solve (V(0,1), W on levels 2-4) takes the same
    iterations to the same lambda with and without the fused coarse cycle."""
    from hicar_b200 import wind, wind_iterative as wi
    res = {}
    for fuse in ("0", "1"):
        monkeypatch.setenv("HICARW_MG_FUSE", fuse)
        wi.finalize_iter_winds()
        wind.reset()
        dom, _, div, _ = _calibrated(case)
        h = wi.handle(dom.nest_indx)
        wi.set_options(wi.WindOptions(tol_rel=1e-9, wind_solver_iterations=3000, precond=_capi.PRECOND_MG,
                                      stall_iters=50, mg_skip_fine_presmooth=True, mg_omega=1.0,
                                      mg_w_levels=(2, 3, 4)))
        dom.set_winds(case.u, case.v, case.w)
        _capi.load().hicarw_reset_solution(h, None)
        wind.calc_divergence(div, dom, use_dqdt=True)
        st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
        lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
        _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
        res[fuse] = (st, lam)
    assert res["1"][0]["status"] == 0
    assert res["1"][0]["iterations"] == res["0"][0]["iterations"]
    np.testing.assert_array_equal(res["1"][1], res["0"][1])


@pytest.mark.parametrize("shape", [(48, 40, 20), (197, 101, 13)])
def test_vcycle_bf16_finest_smoother(shape, monkeypatch):
    """mg_precision = 1: the finest level's post-smoother reads its coefficients
    in BF16 (tensor-copy and register-fed kernels alike, bit-identical) and
    solves the BF16-rounded tridiagonal; against the numpy restatement with the
    same rounding, V(0,1) with W on levels 2-3."""
    import mg_ref
    from hicar_b200 import wind, wind_iterative as wi
    nx, ny, nz = shape
    case = cases.build_case(nx, ny, nz, seed=33, adv_den=True, n_hills=10)
    rng = np.random.default_rng(37)
    x = np.zeros((ny + 2, nz + 2, nx + 2))
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((ny, nz, nx))
    cyc = dict(mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=(2, 3))
    out = {}
    for tma in ("2", "1", "0"):  # both tensor-copy kernels, then the register-fed one
        monkeypatch.setenv("HICARW_MG_TMA", tma)
        wi.finalize_iter_winds()
        wind.reset()
        dom, _, _, _ = _calibrated(case)
        h = wi.handle(dom.nest_indx)
        wi.set_options(wi.WindOptions(mg_precision=1, **cyc))
        y = np.empty_like(x)
        _capi.check(_capi.load().hicarw_apply_precond(h, x.ctypes.data, y.ctypes.data, 0, _capi.MEM_HOST, None), h)
        out[tma] = y
        coefs = _coefs(dom)
    np.testing.assert_array_equal(out["2"], out["0"])
    np.testing.assert_array_equal(out["1"], out["0"])
    want = mg_ref.VCycle(coefs, 1.0, fine_presmooth=False, wlevels=(2, 3), fine_bf16=True)(x[1:-1, 1:-1, 1:-1])
    assert _rel(out["2"][1:-1, 1:-1, 1:-1], want) < 1e-5
    f32 = mg_ref.VCycle(coefs, 1.0, fine_presmooth=False, wlevels=(2, 3))(x[1:-1, 1:-1, 1:-1])
    assert _rel(out["2"][1:-1, 1:-1, 1:-1], f32) > 1e-6  # the rounding is really applied


def test_mg_solve_bf16_finest_smoother(oracle_mod, case):
    """The headline cycle with the BF16 finest-level smoother and FP32 Krylov
    vectors (FP64 lambda) converges to the oracle's lambda at 1e-9."""
    from hicar_b200 import wind, wind_iterative as wi
    dom, opt, div, _ = _calibrated(case)
    h = wi.handle(dom.nest_indx)
    wi.set_options(wi.WindOptions(tol_rel=1e-9, wind_solver_iterations=3000, precond=_capi.PRECOND_MG,
                                  stall_iters=50, mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=(2, 3, 4),
                                  krylov_precision=_capi.KRYLOV_F32_X64, mg_precision=1))
    dom.set_winds(case.u, case.v, case.w)
    _capi.load().hicarw_reset_solution(h, None)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    assert st["status"] == 0 and st["precond"] == _capi.PRECOND_MG
    lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
    _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
    s = oracle_mod.OracleSolver(case.domain)
    s.set_coefs(_coefs(dom), probed=True)
    s.prepare(div.cpu().numpy())
    s.set_vec("x", np.zeros_like(lam))
    s.set_tolerance(1e-10)
    assert s.bicgstab(3000)["status"] == 0
    assert _rel(lam, s.vec("x")) < 1e-5
