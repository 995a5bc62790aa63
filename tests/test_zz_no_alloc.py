"""GPU test of hicarw_residual_norm_noalloc, the residual-norm entry point for
callers that cannot allocate device memory (inside a stream capture, or in a
host model whose device memory is fixed up front).  It must agree with the
library's allocating paths on two calls in a row: the FP64 true residual the
solve reports, and ||rhs - A x|| formed from hicarw_apply_operator, for the
probed operator and for the analytic one (its bottom and top boundary rows
and constant horizontal terms).

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from hicar_b200 import _capi, cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_residual_norm_noalloc_matches_allocating_paths(lib):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hicar_b200 import wind, wind_iterative as wi
    from hicar_b200.domain import DeviceDomain
    wi.finalize_iter_winds()
    wind.reset()
    case = cases.build_case(40, 36, 16, seed=9, adv_den=True, n_hills=6)
    dom = DeviceDomain.from_case(case, "cuda")
    opt = wi.WindOptions(tol_rel=1e-8)
    wi.init_iter_winds(dom, opt)
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    wind.calibrate_projection_operator(dom, opt, div)
    h = wi.handle(dom.nest_indx)
    shape = (dom.ny + 2, dom.nz + 2, dom.nx + 2)
    rng = np.random.default_rng(0)
    b = np.zeros(shape)
    b[1:-1, 1:-1, 1:-1] = rng.standard_normal((dom.ny, dom.nz, dom.nx)) * 1e-3
    # call 1: against the FP64 true residual the allocating solve path reports
    st = _capi.Stats()
    assert lib.hicarw_solve_rhs(h, b.ctypes.data, _capi.MEM_HOST, None, C.byref(st)) >= 0
    lam = torch.empty(shape, dtype=torch.float64, device="cuda")
    assert lib.hicarw_get_lambda(h, lam.data_ptr(), _capi.MEM_DEVICE, None) == 0
    bd = torch.from_numpy(b).cuda()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.hicarw_residual_norm_noalloc(h, lam.data_ptr(), bd.data_ptr(), out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert abs(out.item() - st.true_res) <= 1e-9 * st.true_res
    # call 2 (scratch reused): another x, against hicarw_apply_operator
    x2 = lam * 0.5 + 1e-4
    x2[0], x2[-1], x2[:, 0], x2[:, -1], x2[:, :, 0], x2[:, :, -1] = 0, 0, 0, 0, 0, 0
    assert lib.hicarw_residual_norm_noalloc(h, x2.data_ptr(), bd.data_ptr(), out.data_ptr(), None) == 0
    xh = x2.cpu().numpy()
    y = np.empty(shape)
    assert lib.hicarw_apply_operator(h, xh.ctypes.data, y.ctypes.data, _capi.MEM_HOST, None) == 0
    ref = float(np.linalg.norm(b - y))
    torch.cuda.synchronize()
    assert abs(out.item() - ref) <= 1e-9 * ref
    wi.finalize_iter_winds()
    wind.reset()


def test_residual_norm_noalloc_analytic_operator(lib):
    """The analytic operator of the first solve (before any calibration): two
    calls in a row against ||rhs - A x|| formed from hicarw_apply_operator."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hicar_b200 import wind, wind_iterative as wi
    from hicar_b200.domain import DeviceDomain
    wi.finalize_iter_winds()
    wind.reset()
    case = cases.build_case(37, 29, 11, seed=5, adv_den=True, n_hills=4)
    dom = DeviceDomain.from_case(case, "cuda")
    opt = wi.WindOptions()
    wi.init_iter_winds(dom, opt)
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    wind.calc_divergence(div, dom, use_dqdt=True)
    wi.calc_iter_winds(dom, dom.wind_alpha, div, True)  # builds the analytic coefficients
    h = wi.handle(dom.nest_indx)
    shape = (dom.ny + 2, dom.nz + 2, dom.nx + 2)
    rng = np.random.default_rng(3)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for call in range(2):
        x = rng.standard_normal(shape)
        b = rng.standard_normal(shape)
        xd, bd = torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda()
        assert lib.hicarw_residual_norm_noalloc(h, xd.data_ptr(), bd.data_ptr(), out.data_ptr(), None) == 0
        y = np.empty(shape)
        assert lib.hicarw_apply_operator(h, x.ctypes.data, y.ctypes.data, _capi.MEM_HOST, None) == 0
        ref = float(np.linalg.norm(b - y))
        torch.cuda.synchronize()
        assert abs(out.item() - ref) <= 1e-9 * ref, (call, out.item(), ref)
    wi.finalize_iter_winds()
    wind.reset()
