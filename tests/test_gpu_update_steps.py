"""GPU parity of the steps either side of the solve in update_winds
(calc_w_real, calc_idealized_wgrid, balance_uvw/calc_w, calc_alpha and the
smoothing of alpha) against the oracle's reference-precision restatement:
bit-exact (FP32 in the reference's order of operations, no FMA contraction)."""
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


@pytest.fixture(scope="module", params=[(48, 40, 16), (33, 17, 7)])
def setup(request, oracle_mod):
    nx, ny, nz = request.param
    case = cases.build_case(nx, ny, nz, seed=21, adv_den=True, n_hills=8)
    return case, oracle_mod.OracleSolver(case.domain, "ref")


def _handle(case):
    from hicar_b200 import wind_iterative as wi
    from hicar_b200.domain import DeviceDomain
    dom = DeviceDomain.from_case(case, "cuda")
    wi.init_iter_winds(dom, wi.WindOptions())
    return dom, wi.handle(dom.nest_indx)


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _p(t):
    return t.data_ptr()


def _eq(gpu, ref):
    np.testing.assert_array_equal(gpu.cpu().numpy(), np.asarray(ref, np.float32))


def test_w_real(setup):
    case, s = setup
    dom, h = _handle(case)
    lib = _capi.load()
    rng = np.random.default_rng(1)
    wg = rng.standard_normal(case.w.shape).astype(np.float32)
    u, v = _t(case.u), _t(case.v)
    for w_grid in (None, wg):
        out = torch.empty(case.w.shape, dtype=torch.float32, device="cuda")
        wgt = _t(w_grid) if w_grid is not None else None
        _capi.check(lib.hicarw_calc_w_real(h, _p(u), _p(v), _p(wgt) if wgt is not None else None,
                                           _p(out), _capi.MEM_DEVICE, None), h)
        torch.cuda.synchronize()
        _eq(out, s.w_real(case.u, case.v, w_grid))


def test_idealized_wgrid(setup):
    case, s = setup
    dom, h = _handle(case)
    lib = _capi.load()
    field = np.random.default_rng(2).standard_normal(case.w.shape).astype(np.float32)
    out = torch.full(case.w.shape, 7.0, dtype=torch.float32, device="cuda")
    u, v, f = _t(case.u), _t(case.v), _t(field)
    _capi.check(lib.hicarw_calc_idealized_wgrid(h, _p(u), _p(v), _p(f), _p(out), _capi.MEM_DEVICE, None), h)
    torch.cuda.synchronize()
    _eq(out, s.idealized_wgrid(case.u, case.v, field))


@pytest.mark.parametrize("adv_den", [True, False])
def test_balance_uvw(setup, adv_den):
    case, s = setup
    dom, h = _handle(case)
    lib = _capi.load()
    w, u, v, rho = _t(case.w), _t(case.u), _t(case.v), _t(case.domain.density)
    _capi.check(lib.hicarw_balance_uvw(h, _p(u), _p(v), _p(rho), _p(w), int(adv_den), 1, _capi.MEM_DEVICE, None), h)
    torch.cuda.synchronize()
    _eq(w, s.balance_uvw(case.u, case.v, case.w, adv_den=adv_den, use_dqdt=True))


def test_calc_alpha_and_smoothing(setup):
    case, s = setup
    dom, h = _handle(case)
    lib = _capi.load()
    rng = np.random.default_rng(3)
    fr = np.exp(rng.uniform(np.log(0.05), np.log(20.0), case.w.shape)).astype(np.float32)
    a = torch.empty(case.w.shape, dtype=torch.float32, device="cuda")
    frt = _t(fr)
    _capi.check(lib.hicarw_calc_alpha(h, _p(frt), _p(a), 2, _capi.MEM_DEVICE, None), h)
    torch.cuda.synchronize()
    ref = s.calc_alpha(fr, halo=2)
    _eq(a, ref)
    _capi.check(lib.hicarw_smooth_alpha(h, _p(a), 2, 3, _capi.MEM_DEVICE, None), h)
    torch.cuda.synchronize()
    _eq(a, s.smooth_array(ref, 2, 3))


def test_update_stability(setup):
    """update_stability on the device against the oracle: the bulk Richardson
    number bit-exact; the Froude number bit-exact in every cell whose wind
    direction is not within 1e-4 degree of a 5-degree sector edge (atan2f is not
    correctly rounded, so such a cell may take the neighbouring sector), and
    the Froude branch switched off leaves 0.1 everywhere."""
    case, s = setup
    if case.domain.nz < 5:
        pytest.skip("update_stability reads the wind at level 5")
    dom, h = _handle(case)
    theta, ft = cases.stability_inputs(case, seed=5)
    ref_fr, ref_ri = s.update_stability(case.u, case.v, case.domain.z, theta, ft)
    fr = torch.empty(case.w.shape, dtype=torch.float32, device="cuda")
    ri = torch.empty_like(fr)
    from hicar_b200 import wind
    wind.update_stability(dom, _t(case.domain.z), _t(theta), fr, ri, froude_terrain=_t(ft))
    torch.cuda.synchronize()
    _eq(ri, ref_ri)
    um = 0.5 * (case.u[:, :, :-1].astype(np.float64) + case.u[:, :, 1:])
    vm = 0.5 * (case.v[:-1].astype(np.float64) + case.v[1:])
    wd = np.degrees(np.arctan2(-um, -vm)) % 360.0
    edge = np.abs(wd / 5.0 - np.round(wd / 5.0)) * 5.0 < 1e-4
    diff = fr.cpu().numpy() != ref_fr
    assert not (diff & ~edge).any(), int((diff & ~edge).sum())
    wind.update_stability(dom, _t(case.domain.z), _t(theta), fr, ri, froude_terrain=None, froude_mode=False)
    torch.cuda.synchronize()
    assert bool((fr == 0.1).all())
