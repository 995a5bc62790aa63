"""GPU tests of the composite learned preconditioner HICARW_PRECOND_MG_LEARNED,
z = M(r) + theta U(r'), r' = r - A M(r): the V-cycle, then the U-Net's estimate
of the error left in the residual the V-cycle leaves, with the minimal-residual
step theta, inside FGMRES.

* The composite applied by the library equals its parts composed through the
  C ABI (V-cycle, operator, U-Net apply, the step), and leaves no larger a
  residual than the V-cycle alone.
* FGMRES with the composite converges to the oracle's lambda.
* The training-pair generator logs one pair per requested iterate of the
  plain solver, with finite, non-zero targets of the network's output shape.
* A/B against the method without the network (FGMRES + the same V-cycle):
  the iteration counts of both are reported, and the composite with the
  shipped parameters needs no more iterations than the V-cycle alone.

Collected after the other solver tests (the allocation-free entry point's
file comes last)."""
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


def _net(dom, trained=True):
    from hicar_b200 import learned as L
    from hicar_b200.train_unet import COMPOSITE_WEIGHTS, load_params
    net = L.UNet(dom.nx, dom.ny, dom.nz, seed=5)
    if trained and os.path.exists(COMPOSITE_WEIGHTS):
        net.set_params(torch.from_numpy(load_params(COMPOSITE_WEIGHTS)))
    return net


def test_composite_equals_its_parts():
    from hicar_b200 import learned as L, wind_iterative as wi
    case = cases.build_case(40, 36, 12, seed=31, adv_den=True, n_hills=6)
    dom, h = L.calibrated_handle(case)
    net = _net(dom, trained=False)
    net.attach(h)
    lib = _capi.load()
    wi.set_options(wi.WindOptions(solver=_capi.SOLVER_FGMRES, precond=_capi.PRECOND_MG_LEARNED, **L.MG_CYCLE))
    shape = (dom.ny + 2, dom.nz + 2, dom.nx + 2)
    r = torch.zeros(shape, dtype=torch.float64, device="cuda")
    r[1:-1, 1:-1, 1:-1] = torch.randn((dom.ny, dom.nz, dom.nx), generator=torch.Generator().manual_seed(3),
                                      dtype=torch.float64).cuda()
    z = torch.empty_like(r)
    _capi.check(lib.hicarw_apply_precond(h, r.data_ptr(), z.data_ptr(), -1, _capi.MEM_DEVICE, None), h)
    z1 = torch.empty_like(r)
    _capi.check(lib.hicarw_apply_precond(h, r.data_ptr(), z1.data_ptr(), 0, _capi.MEM_DEVICE, None), h)
    az = torch.empty_like(r)
    _capi.check(lib.hicarw_apply_operator(h, z1.data_ptr(), az.data_ptr(), _capi.MEM_DEVICE, None), h)
    rp = r - az
    u = net.apply(h, rp)
    au = torch.empty_like(r)
    _capi.check(lib.hicarw_apply_operator(h, u.data_ptr(), au.data_ptr(), _capi.MEM_DEVICE, None), h)
    theta = float((rp * au).sum() / (au * au).sum())  # the minimal-residual step along u
    want = z1 + theta * u
    torch.cuda.synchronize()
    assert _rel(z.cpu().numpy(), want.cpu().numpy()) < 1e-12
    # the composite leaves no larger a residual than the V-cycle alone
    _capi.check(lib.hicarw_apply_operator(h, z.data_ptr(), az.data_ptr(), _capi.MEM_DEVICE, None), h)
    assert float((r - az).norm()) <= float(rp.norm()) * (1.0 + 1e-12)
    lib.hicarw_set_learned_precond(h, None)


def test_composite_pairs_are_consistent():
    """One pair per logged iterate, targets e' coef_A / rms(r') of the
    network's output shape, finite and non-zero."""
    from hicar_b200 import learned as L
    case = cases.build_case(32, 32, 12, seed=1001, adv_den=True, n_hills=6)
    net = L.UNet(32, 32, 12, seed=5)
    pairs = L.composite_pairs(case, net, ks=(1, 8, 64))
    assert len(pairs) == 3
    for x0, target in pairs:
        assert target.shape == (32, 12, 32)
        assert torch.isfinite(target).all() and float(target.abs().max()) > 0.0


def _fgmres_solve(dom, h, case, precond, tol=1e-8):
    from hicar_b200 import learned as L, wind, wind_iterative as wi
    wi.set_options(wi.WindOptions(tol_rel=tol, wind_solver_iterations=3000, solver=_capi.SOLVER_FGMRES,
                                  precond=precond, stall_iters=200, fgmres_restart=30, **L.MG_CYCLE))
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    dom.set_winds(case.u, case.v, case.w)
    _capi.load().hicarw_reset_solution(h, None)
    wind.calc_divergence(div, dom, use_dqdt=True)
    st = wi.calc_iter_winds(dom, dom.wind_alpha, div, True)
    lam = np.empty((dom.ny + 2, dom.nz + 2, dom.nx + 2))
    _capi.load().hicarw_get_lambda(h, lam.ctypes.data, _capi.MEM_HOST, None)
    return st, lam, div


def test_composite_fgmres_matches_oracle_and_ab(oracle_mod):
    from hicar_b200 import learned as L
    case = cases.build_case(96, 80, 24, seed=7, adv_den=True, n_hills=8, alpha="smooth")
    dom, h = L.calibrated_handle(case)
    net = _net(dom)
    net.attach(h)
    st_l, lam_l, div = _fgmres_solve(dom, h, case, _capi.PRECOND_MG_LEARNED)
    st_m, lam_m, _ = _fgmres_solve(dom, h, case, _capi.PRECOND_MG)
    assert st_l["status"] == 0 and st_l["precond"] == _capi.PRECOND_MG_LEARNED, st_l
    assert st_m["status"] == 0 and st_m["precond"] == _capi.PRECOND_MG, st_m
    coefs = np.empty((15, dom.ny, dom.nz, dom.nx), np.float32)
    _capi.check(_capi.load().hicarw_get_coefs(h, coefs.ctypes.data, _capi.MEM_HOST, None), h)
    s = oracle_mod.OracleSolver(case.domain)
    s.set_coefs(coefs, probed=True)
    s.prepare(div.cpu().numpy())
    s.set_vec("x", np.zeros_like(lam_l))
    s.set_tolerance(1e-10)
    assert s.bicgstab(5000)["status"] == 0
    assert _rel(lam_l, s.vec("x")) < 1e-5
    assert _rel(lam_m, s.vec("x")) < 1e-5
    print(f"FGMRES(30) iterations to 1e-8: V-cycle + U-Net {st_l['iterations']}, V-cycle {st_m['iterations']}")
    from hicar_b200.train_unet import COMPOSITE_WEIGHTS
    if os.path.exists(COMPOSITE_WEIGHTS):
        assert st_l["iterations"] <= st_m["iterations"], (st_l["iterations"], st_m["iterations"])
