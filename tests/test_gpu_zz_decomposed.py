"""GPU test of the decomposed solve (hicarw_dist_* through hicar_b200.decomp):
the ranks of a 2 x 1 and a 2 x 2 x-y decomposition run as library handles on
this one GPU, their schedules interleaved in one process (run_local: the face
exchange by copies, the allreduce by a sum; no kernel waits for another).
The assembled lambda must equal the one-handle solve of the whole domain with
the same probed operator and right-hand side, for the reference's block
Jacobi-Richardson preconditioner and for block V-cycles, and every rank must
end with the same status and iteration count.

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


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("px,py,precond", [(2, 1, _capi.PRECOND_JACOBI), (2, 2, _capi.PRECOND_JACOBI),
                                          (2, 2, _capi.PRECOND_MG)])
def test_decomposed_solve_matches_one_rank(px, py, precond):
    import ctypes as C

    from hicar_b200 import decomp, learned as L, wind_iterative as wi
    from hicar_b200.domain import DeviceDomain
    nx, ny, nz = 64, 48, 16
    case = cases.build_case(nx, ny, nz, seed=51, adv_den=True, n_hills=6)
    dom, h = L.calibrated_handle(case)
    lib = _capi.load()
    coefs = torch.empty((15, ny, nz, nx), dtype=torch.float32, device="cuda")
    _capi.check(lib.hicarw_get_coefs(h, coefs.data_ptr(), _capi.MEM_DEVICE, None), h)
    rng = np.random.default_rng(7)
    rhs = np.zeros((ny + 2, nz + 2, nx + 2))
    rhs[1:-1, 1:-1, 1:-1] = rng.standard_normal((ny, nz, nx))
    opt = wi.WindOptions(tol_rel=1e-10, wind_solver_iterations=3000, precond=precond)
    wi.set_options(opt)
    lib.hicarw_reset_solution(h, None)
    st = _capi.Stats()
    assert lib.hicarw_solve_rhs(h, rhs.ctypes.data, _capi.MEM_HOST, None, C.byref(st)) == 0
    lam_ref = np.empty_like(rhs)
    _capi.check(lib.hicarw_get_lambda(h, lam_ref.ctypes.data, _capi.MEM_HOST, None), h)

    dec = decomp.Decomposition(nx, ny, px, py)
    ranks, schedules = [], []
    for q in range(dec.size):
        ld = DeviceDomain.from_case(decomp.local_case(case, dec, q), "cuda")
        r = decomp.CudaRank(ld, dec.interior(q, coefs).contiguous(), dec.edges(q), options=opt)
        ranks.append(r)
        schedules.append(decomp.rank_schedule(r, dec.neighbors(q), np.ascontiguousarray(dec.local(q, rhs)), 3000))
    stats = decomp.run_local(schedules, dec)
    lam = np.zeros_like(rhs)
    for q, r in enumerate(ranks):
        i0, i1, j0, j1 = dec.block(q)
        lam[j0:j1 + 1, 1:-1, i0:i1 + 1] = r.lam().cpu().numpy()[1:-1, 1:-1, 1:-1]
        r.close()
    print(f"{px}x{py} ranks, precond {precond}: {stats[0]['iterations']} iterations "
          f"(one rank {st.iterations}), lambda error {_rel(lam, lam_ref):.2e}")
    assert all(s_["status"] == 0 for s_ in stats), stats
    assert len({s_["iterations"] for s_ in stats}) == 1
    assert _rel(lam[1:-1, 1:-1, 1:-1], lam_ref[1:-1, 1:-1, 1:-1]) < 1e-7
