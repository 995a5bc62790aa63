"""CPU tests of the oracle (the checker) against known answers.

The reference ships no golden vector for this path, so the oracle is pinned
by properties the reference's own algorithm guarantees:
  * the probed operator IS the composition 2 D o G (wind_iterative.F90:1078-1094);
  * a manufactured lambda* is recovered from b = A lambda*;
  * the reference unit test's assertion (tests/unit/test_wind_iterative.F90:139-152):
    the solve reduces max|div| on its flat-plane cos/sin wind field;
  * the calibrated projection removes the divergence to solver tolerance;
  * reference precision and the all-FP64 build agree.
"""
import numpy as np
import pytest

from hicar_b200 import cases


def _interior_random(s, rng, smooth=False):
    lam = np.zeros((s.ny + 2, s.nz + 2, s.nx + 2))
    inner = rng.standard_normal((s.ny, s.nz, s.nx))
    if smooth:
        for ax in range(3):
            inner = 0.5 * (inner + np.roll(inner, 1, axis=ax))
    lam[1:-1, 1:-1, 1:-1] = inner
    return lam


@pytest.fixture(scope="module")
def c1():
    return cases.build_case(24, 20, 10, seed=3, adv_den=True, n_hills=6)


def test_generator_metrics(c1):
    d = c1.domain
    assert d.jacobian.min() > 0.0
    assert d.jacobian_w.shape == (d.ny, d.nz, d.nx)
    assert d.dzdx_u.shape == (d.ny, d.nz, d.nx + 1)
    assert d.dzdy_v.shape == (d.ny + 1, d.nz, d.nx)
    assert np.all(d.jacobian_w[:, -1, :] == 1.0)  # domain_obj.F90:2022
    nom = cases.nominal_levels(d.nz)
    assert np.isclose(d.dz_levels.sum(), d.terrain.max() + nom.sum(), rtol=1e-5)


def test_probe_leakage_zero_and_composition(oracle_mod, c1):
    """A = 2 D o G: the probed 15-point operator applied to any lambda equals
    2 * div(G(lambda)) evaluated directly (FP32 rounding tolerance)."""
    s = oracle_mod.OracleSolver(c1.domain)
    u, v, w = (np.ascontiguousarray(a).copy() for a in (c1.u, c1.v, c1.w))
    s.set_alpha(c1.alpha)
    leak = s.calibrate(True, u, v, w)
    assert leak == 0.0
    # calibration restores the caller's winds
    assert np.array_equal(u, c1.u) and np.array_equal(w, c1.w)
    rng = np.random.default_rng(0)
    lam = _interior_random(s, rng)
    y = s.spmv(lam)
    s.set_vec("x", lam)
    uz, vz, wz = (np.zeros_like(a) for a in (c1.u, c1.v, c1.w))
    s.updated_winds(True, uz, vz, wz)
    direct = 2.0 * s.divergence(uz, vz, wz, adv_den=True).astype(np.float64)
    got = y[1:-1, 1:-1, 1:-1]
    err = np.linalg.norm(got - direct) / np.linalg.norm(direct)
    assert err < 1e-5, err
    # boundary rows are identity rows
    assert np.array_equal(y[0], lam[0]) and np.array_equal(y[:, 0], lam[:, 0])


def test_manufactured_solution(oracle_mod, c1):
    s = oracle_mod.OracleSolver(c1.domain)
    s.build_analytic(c1.alpha)
    u, v, w = (np.ascontiguousarray(a).copy() for a in (c1.u, c1.v, c1.w))
    s.calibrate(True, u, v, w)
    rng = np.random.default_rng(1)
    lam = _interior_random(s, rng, smooth=True)
    b = s.spmv(lam)
    s.prepare(np.zeros((s.ny, s.nz, s.nx), np.float32))
    s.set_vec("rhs", b)
    s.set_vec("x", np.zeros_like(b))
    # 1e-9: tighter targets meet the reference's absolute breakdown guard <t,t> < 1e-30
    s.set_tolerance(1e-9, 1e-30)
    st = s.bicgstab(5000)
    assert st["status"] == 0
    x = s.vec("x")
    err = np.linalg.norm(x - lam) / np.linalg.norm(lam)
    assert err < 1e-5, err


def test_reference_unit_test_assertion(oracle_mod):
    """tests/unit/test_wind_iterative.F90:118-152 on its flat plane set-up."""
    uc = cases.unit_test_case(32, 24, 20)
    s = oracle_mod.OracleSolver(uc.domain)
    u, v, w = uc.u.copy(), uc.v.copy(), uc.w.copy()
    div0 = s.divergence(u, v, w, adv_den=False)
    rc, st = s.calc_iter_winds(uc.alpha, div0, False, u, v, w)
    assert rc == 0 and st["status"] == 0
    div1 = s.divergence(u, v, w, adv_den=False)
    assert not np.isnan(div1).any()
    assert np.abs(div1).max() < np.abs(div0).max()


def test_calibrated_projection_removes_divergence(oracle_mod, c1):
    s, u, v, w, st1, st2, leak = oracle_mod.update_winds_first(c1)
    assert st1["status"] == 0 and st2["status"] == 0
    div0 = s.divergence(c1.u, c1.v, c1.w, adv_den=True)
    div1 = s.divergence(u, v, w, adv_den=True)
    assert np.abs(div1).max() < 1e-3 * np.abs(div0).max()


def test_fp32_fields_vs_fp64_oracle(oracle_mod, c1):
    s32, u32, v32, w32, *_ = oracle_mod.update_winds_first(c1, "ref", tol_rel=1e-10)
    s64, u64, v64, w64, *_ = oracle_mod.update_winds_first(c1, "f64", tol_rel=1e-10)
    for a, b in ((u32, u64), (v32, v64), (w32, w64)):
        e = np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b)
        assert e < 1e-4, e


def test_divergence_linear(oracle_mod, c1):
    s = oracle_mod.OracleSolver(c1.domain)
    rng = np.random.default_rng(2)
    u2, v2, w2 = (rng.standard_normal(a.shape).astype(np.float32) for a in (c1.u, c1.v, c1.w))
    d1 = s.divergence(c1.u, c1.v, c1.w).astype(np.float64)
    d2 = s.divergence(u2, v2, w2).astype(np.float64)
    d12 = s.divergence(c1.u + u2, c1.v + v2, c1.w + w2).astype(np.float64)
    assert np.linalg.norm(d12 - d1 - d2) / np.linalg.norm(d12) < 1e-5


def test_retry_bumps_sweeps(oracle_mod, c1):
    """Adaptive preconditioner retry (wind_iterative.F90:479-503): with an
    iteration cap too small to converge, the solve is retried with more sweeps."""
    s = oracle_mod.OracleSolver(c1.domain, max_iters=3)
    u, v, w = (np.ascontiguousarray(a).copy() for a in (c1.u, c1.v, c1.w))
    div = s.divergence(u, v, w)
    rc, st = s.calc_iter_winds(c1.alpha, div, True, u, v, w)
    assert st["status"] == 1
    assert st["retries"] >= 1 and st["sweeps"] > 2


@pytest.mark.parametrize("shape", [(17, 13, 5), (5, 7, 2)])
def test_odd_sizes(oracle_mod, shape):
    nx, ny, nz = shape
    c = cases.build_case(nx, ny, nz, seed=11, n_hills=3)
    s, u, v, w, st1, st2, leak = oracle_mod.update_winds_first(c)
    assert st2["status"] == 0 and leak == 0.0
    assert np.isfinite(u).all() and np.isfinite(v).all() and np.isfinite(w).all()
