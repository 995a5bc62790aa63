"""GPU tests of the batched solver (hicarw_batch_*): one graph launch with a
device-driven loop per subdomain must give, for every subdomain of an uneven
batch, the same iterations, lambda and corrected winds as that subdomain's own
hicarw_calc_iter_winds (the same kernels in the same order: bit-exact), for
every lane / chunk configuration; the autotuner picks a configuration; a
stalled multigrid solve falls back to the reference solve."""
import ctypes as C

import numpy as np
import pytest

from hicar_b200 import _capi, cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SIZES = [(40, 32, 10), (64, 48, 12), (33, 17, 8), (72, 40, 16), (48, 48, 10)]


@pytest.fixture(autouse=True)
def _gpu(lib):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _cases():
    return [cases.build_case(nx, ny, nz, seed=50 + i, adv_den=True, n_hills=6) for i, (nx, ny, nz) in enumerate(SIZES)]


def _single(bs, i):
    """Subdomain i solved alone through hicarw_calc_iter_winds from the saved winds."""
    from hicar_b200.domain import ptr
    lib = _capi.load()
    h, dom = bs.handles[i], bs.domains[i]
    dom.set_winds(*bs.saved[i])
    bs.divergence()
    lib.hicarw_reset_solution(h, C.c_void_p(bs.stream))
    st = _capi.Stats()
    rc = lib.hicarw_calc_iter_winds(h, ptr(dom.wind_alpha), ptr(bs.divs[i]), ptr(dom.density), 1, ptr(dom.u_dqdt),
                                    ptr(dom.v_dqdt), ptr(dom.w_dqdt), _capi.MEM_DEVICE, C.c_void_p(bs.stream),
                                    C.byref(st))
    _capi.check(rc, h)
    return st.as_dict(), bs.lambda_of(i).cpu(), [a.clone().cpu() for a in (dom.u_dqdt, dom.v_dqdt, dom.w_dqdt)]


@pytest.fixture(scope="module")
def solver():
    from hicar_b200.batch import BatchSolver
    bs = BatchSolver(_cases())
    yield bs
    bs.close()


@pytest.mark.parametrize("lanes,chunk", [(0, 4), (1, 2), (2, 8)])
def test_batch_matches_single_solves(solver, lanes, chunk):
    bs = solver
    bs.configure(lanes, chunk)
    stats = bs.step()
    lam_b = [bs.lambda_of(i).cpu() for i in range(bs.n)]
    lat = bs.latencies()
    assert (lat > 0).all() and np.isfinite(lat).all()
    winds_b = [[a.clone().cpu() for a in (d.u_dqdt, d.v_dqdt, d.w_dqdt)] for d in bs.domains]
    for i in range(bs.n):
        st, lam, winds = _single(bs, i)
        assert stats[i]["status"] == 0 and st["status"] == 0
        assert stats[i]["precond"] == _capi.PRECOND_MG
        assert stats[i]["iterations"] == st["iterations"]
        assert stats[i]["true_res"] <= 1.01 * stats[i]["target"]
        assert torch.equal(lam_b[i], lam)
        for a, b in zip(winds_b[i], winds):
            assert torch.equal(a, b)


def test_batch_autotune(solver):
    bs = solver
    best = bs.autotune()
    lanes, chunk = bs.config()
    assert best > 0.0
    assert lanes in (1, 4) and chunk in (4, 8)
    stats = bs.step()
    assert all(s["status"] == 0 for s in stats)
    st, lam, _ = _single(bs, 3)
    bs.step()
    assert torch.equal(bs.lambda_of(3).cpu(), lam)


def test_batch_stall_falls_back():
    """A useless multigrid damping (omega = 3) stalls the preconditioned solves;
    every subdomain falls back to the reference Jacobi solve (status 3)."""
    from hicar_b200.batch import BatchSolver
    from hicar_b200.wind_iterative import WindOptions
    opts = WindOptions(tol_rel=1e-6, wind_solver_iterations=400, precond=_capi.PRECOND_MG, stall_iters=10,
                       mg_omega=3.0)
    bs = BatchSolver(_cases()[:2], options=opts)
    try:
        stats = bs.step()
        for s in stats:
            assert s["status"] == _capi.HICARW_FELL_BACK
            assert s["true_res"] <= 1.5 * s["target"]
        assert np.isfinite(bs.lambda_of(0).cpu().numpy()).all()
    finally:
        bs.close()


def test_batch_mixes_fgmres_and_learned_with_bicgstab():
    """One batch holding a Jacobi BiCGStab ("plain") subdomain, an MG BiCGStab one,
    an MG-FGMRES one and a learned-FGMRES one: each matches its own single solve
    (same kernels, same order: bit-exact)."""
    from hicar_b200 import learned as L
    from hicar_b200.batch import BatchSolver
    from hicar_b200.train_unet import load_params
    from hicar_b200.wind_iterative import WindOptions
    cs = _cases()[:4]
    bs = BatchSolver(cs)
    try:
        lib = _capi.load()
        opts = [WindOptions(tol_rel=1e-6, wind_solver_iterations=3000),
                WindOptions(tol_rel=1e-6, wind_solver_iterations=3000, precond=_capi.PRECOND_MG, stall_iters=50),
                WindOptions(tol_rel=1e-6, wind_solver_iterations=3000, precond=_capi.PRECOND_MG,
                            solver=_capi.SOLVER_FGMRES),
                WindOptions(tol_rel=1e-6, wind_solver_iterations=3000, precond=_capi.PRECOND_LEARNED,
                            solver=_capi.SOLVER_FGMRES, stall_iters=100)]
        nets = []
        for h, o, d in zip(bs.handles, opts, bs.domains):
            _capi.check(lib.hicarw_set_options(h, C.byref(o.to_c())), h)
            if o.precond == _capi.PRECOND_LEARNED:
                net = L.UNet(d.nx, d.ny, d.nz)
                net.set_params(torch.from_numpy(load_params()))
                net.attach(h)
                nets.append(net)
        stats = bs.step()
        lam_b = [bs.lambda_of(i).cpu() for i in range(bs.n)]
        kinds = [s["precond"] for s in stats]
        assert kinds == [_capi.PRECOND_JACOBI, _capi.PRECOND_MG, _capi.PRECOND_MG, _capi.PRECOND_LEARNED]
        for i in range(bs.n):
            st, lam, _ = _single(bs, i)
            assert stats[i]["status"] == 0 and st["status"] == 0
            assert stats[i]["iterations"] == st["iterations"]
            assert stats[i]["true_res"] <= 1.05 * stats[i]["target"]
            assert torch.equal(lam_b[i], lam)
    finally:
        bs.close()
