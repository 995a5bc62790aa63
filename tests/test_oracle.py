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


# ---- the steps either side of the solve in update_winds ----------------------
def test_balance_uvw_closes_the_divergence(oracle_mod, c1):
    """balance_uvw's w makes the full 3-D divergence vanish: the vertical flux
    difference of calc_w cancels the horizontal divergence level by level."""
    s = oracle_mod.OracleSolver(c1.domain, "f64")
    for adv in (True, False):
        dh = s.divergence(c1.u, c1.v, c1.w, adv_den=adv, horz_only=True, use_dqdt=True)
        w = s.balance_uvw(c1.u, c1.v, c1.w, adv_den=adv, use_dqdt=True)
        full = s.divergence(c1.u, c1.v, w, adv_den=adv, horz_only=False, use_dqdt=True)
        assert np.abs(full).max() <= 1e-9 * np.abs(dh).max()


def test_w_real_and_idealized_wgrid(oracle_mod, c1):
    s = oracle_mod.OracleSolver(c1.domain, "f64")
    d = c1.domain
    rng = np.random.default_rng(5)
    wg = rng.standard_normal(c1.w.shape)
    # w_grid part alone (u = v = 0): mean of w_grid * J over the two levels, zero below
    zu, zv = np.zeros_like(c1.u), np.zeros_like(c1.v)
    wr = s.w_real(zu, zv, wg)
    wj = wg * d.jacobian_w.astype(np.float64)
    ref = 0.5 * wj
    ref[:, 1:, :] += 0.5 * wj[:, :-1, :]
    np.testing.assert_allclose(wr, ref, rtol=1e-12, atol=1e-12)
    # the u/v part: face means of u dz/dx and v dz/dy
    wr2 = s.w_real(c1.u, c1.v)
    uu = c1.u.astype(np.float64) * d.dzdx_u
    vv = c1.v.astype(np.float64) * d.dzdy_v
    ref2 = 0.5 * (uu[:, :, :-1] + uu[:, :, 1:]) + 0.5 * (vv[:-1] + vv[1:])
    np.testing.assert_allclose(wr2, ref2, rtol=1e-12, atol=1e-12)
    # idealized w_grid: staggered (w_real_field - w_real(u, v, 0)) / J_w, zero on top
    field = rng.standard_normal(c1.w.shape)
    w = s.idealized_wgrid(c1.u, c1.v, field)
    t = field - wr2
    dz = d.advection_dz.astype(np.float64)
    stag = (t[:, :-1] * dz[:, 1:] + t[:, 1:] * dz[:, :-1]) / (dz[:, :-1] + dz[:, 1:]) / d.jacobian_w[:, :-1]
    np.testing.assert_allclose(w[:, :-1], stag, rtol=1e-12, atol=1e-12)
    assert not w[:, -1].any()


def test_calc_alpha_and_smoothing(oracle_mod, c1):
    s = oracle_mod.OracleSolver(c1.domain, "f64")
    rng = np.random.default_rng(6)
    fr = np.exp(rng.uniform(np.log(0.05), np.log(20.0), c1.w.shape))
    a = s.calc_alpha(fr, halo=2)
    p = np.maximum((1.0 / fr) ** 4, 1e-5)
    ref = np.clip(np.sqrt(np.maximum(1.0 - 0.5 * p * (np.sqrt(1.0 + 4.0 / p) - 1.0), 1e-5)), 0.2, 2.0)
    ref[:, -1, :] = 0.2
    ny, nx = a.shape[0], a.shape[2]
    np.testing.assert_allclose(a[2:ny - 2, :, 2:nx - 2], ref[2:ny - 2, :, 2:nx - 2], rtol=1e-12)
    # halo rows / columns repeat the first tile row / column (south, west, north, east)
    np.testing.assert_array_equal(a[0], a[2])
    np.testing.assert_array_equal(a[:, :, 1], a[:, :, 2])
    np.testing.assert_array_equal(a[-1], a[-3])
    np.testing.assert_array_equal(a[:, :, -2], a[:, :, -3])
    # smoothing: constants are fixed points; an interior spike spreads over the box
    c = np.full(c1.w.shape, 0.7)
    np.testing.assert_allclose(s.smooth_array(c, 2, 3), c, rtol=1e-14)
    spike = np.zeros(c1.w.shape)
    spike[10, 3, 12] = 25.0
    sm = s.smooth_array(spike, 2, 1)
    assert sm[8:13, 3, 10:15] == pytest.approx(np.ones((5, 5)))
    assert sm.sum() == pytest.approx(25.0)


def test_update_stability_known_answers(oracle_mod, c1):
    """update_stability (wind.F90:1421-1565) on a uniform wind and a linear
    potential-temperature profile: the wind blows from 92.5 degrees, so every
    cell takes the blocking height of sector int(92.5/5) + 1 = 19 (a wind from
    exactly 90 degrees lands in sector 18: the reference's rad2deg,
    57.2957779371, is below 180/pi, so 90 degrees reads 89.9999975); the local
    Brunt-Vaisala frequency is g dtheta/dz / theta_surf; the bulk Richardson
    number uses the column between the surface and the level ~100 m up and the
    wind at level 5; the top level keeps Fr = 0.1 and Ri = 10; with the Froude
    branch off every Froude number is 0.1."""
    d = c1.domain
    s = oracle_mod.OracleSolver(d, "f64")
    U0 = 7.5
    ang = np.radians(92.5)
    u = np.full(c1.u.shape, -U0 * np.sin(ang))
    v = np.full(c1.v.shape, -U0 * np.cos(ang))
    z = d.z.astype(np.float64)
    theta = 290.0 + 0.005 * z
    ft = np.full((72, d.ny, d.nz, d.nx), 1.0e6)
    ft[18] = 800.0
    fr, ri = s.update_stability(u, v, z, theta, ft)
    g = 9.81
    n2 = g * (theta[:, 1:, :] - theta[:, :-1, :]) / ((z[:, 1:, :] - z[:, :-1, :]) * theta[:, :1, :])
    np.testing.assert_allclose(fr[:, :-1, :], U0 / (800.0 * np.sqrt(n2)), rtol=1e-10)
    np.testing.assert_array_equal(fr[:, -1, :], 0.1)
    # bulk Ri: Ri_k_max = the last level within 100 m of the surface (at least 2)
    rk = np.argmax(z - z[:, :1, :] > 100.0, axis=1)  # first level above 100 m (0-based)
    rk = np.maximum(rk - 1, 1)
    zt = np.take_along_axis(z, rk[:, None, :], axis=1)[:, 0, :]
    tt = np.take_along_axis(theta, rk[:, None, :], axis=1)[:, 0, :]
    nb = g * (tt - theta[:, 0, :]) / ((zt - z[:, 0, :]) * (tt + theta[:, 0, :]) / 2.0)
    ri_ref = nb / (U0 / (zt - z[:, 0, :])) ** 2
    np.testing.assert_allclose(ri[:, :-1, :], np.broadcast_to(ri_ref[:, None, :], ri[:, :-1, :].shape), rtol=1e-10)
    np.testing.assert_array_equal(ri[:, -1, :], 10.0)
    fr0, _ = s.update_stability(u, v, z, theta, ft, froude_mode=False)
    np.testing.assert_array_equal(fr0, 0.1)
