"""Seeded synthetic HICAR domains for the wind solver.

This module plays the part of HICAR's domain object: it produces the terrain,
vertical levels, metric terms, density and initial winds that the wind solver
reads from ``domain%vars_3d``.  The metric arithmetic restates HICAR's
Gal-Chen set-up at one rank (``setup_simple_z``,
src/objects/domain_obj.F90:1933-2056, with ``max_level = nz``) and the slope
set-up (``setup_dzdxy``, domain_obj.F90:2195-2265) in FP32;
``advection_dz(:,k,:) = dz_levels(k)`` follows domain_obj.F90:2090-2092.
Map factors are 1 (``use_map_factors = .False.``, domain_obj.F90:105-110).

Array layout: numpy C order with shape (ny, nz, nx) — identical in memory to
the Fortran arrays ``(1:nx, 1:nz, 1:ny)`` (i fastest, then k, then j).
u is (ny, nz, nx+1), v is (ny+1, nz, nx), 2-D fields are (ny, nx).

Generator rules (pinned here; the same arrays feed the CPU oracle and the GPU):
  * terrain: sum of ``n_hills`` Gaussian hills, centres U over the domain,
    heights U[200, 2000] m, half-widths U[1, 10] km, sigma = hw / sqrt(2 ln 2);
  * nominal levels dz_k = min(20 * 1.1**(k-1), 500) m.  Gal-Chen needs the
    column top above every hill top, so the levels are scaled by
    s = (max(terrain) + sum(dz)) / sum(dz): the column top is max(terrain) plus
    the nominal column depth, and ``jacobian = (H - h) / H`` stays positive;
  * winds: log profile S * ln(z_agl / z0) / ln(z_ref / z0), z0 = 0.1 m,
    z_ref = 100 m, speed S ~ U[5, 15] m/s, direction ~ U[0, 2 pi), plus N(0, 1)
    noise on u and v; w = 0;
  * density: 1 (``adv_den`` off) or 1.2 * exp(-z / 8000) on mass levels;
  * alpha: constant 1, or a smooth seeded stability field mapped to [0.3, 1.0].
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

F32 = np.float32


@dataclasses.dataclass
class Domain:
    nx: int
    ny: int
    nz: int
    dx: float
    terrain: np.ndarray          # (ny, nx)
    dz_levels: np.ndarray        # (nz,)
    jacobian: np.ndarray         # (ny, nz, nx)
    jacobian_u: np.ndarray       # (ny, nz, nx+1)
    jacobian_v: np.ndarray       # (ny+1, nz, nx)
    jacobian_w: np.ndarray       # (ny, nz, nx)
    dzdx: np.ndarray
    dzdy: np.ndarray
    dzdx_u: np.ndarray           # (ny, nz, nx+1)
    dzdy_v: np.ndarray           # (ny+1, nz, nx)
    advection_dz: np.ndarray     # (ny, nz, nx)
    neighbor_terrain: np.ndarray  # (ny, nx)
    density: np.ndarray          # (ny, nz, nx)
    z: np.ndarray                # mass-level heights (ny, nz, nx)
    mapfac_mx_u: np.ndarray      # (ny, nx+1)
    mapfac_my_v: np.ndarray      # (ny+1, nx)
    mapfac_my_u: np.ndarray      # (ny, nx+1)
    mapfac_mx_v: np.ndarray      # (ny+1, nx)
    mapfac_mxy: np.ndarray       # (ny, nx)
    seed: int = 0

    @property
    def ncell(self) -> int:
        return self.nx * self.ny * self.nz


@dataclasses.dataclass
class Case:
    domain: Domain
    u: np.ndarray      # (ny, nz, nx+1)  u%dqdt_3d
    v: np.ndarray      # (ny+1, nz, nx)  v%dqdt_3d
    w: np.ndarray      # (ny, nz, nx)    w%dqdt_3d (grid-relative w predictor)
    alpha: np.ndarray  # (ny, nz, nx)
    adv_den: bool
    name: str = ""


def nominal_levels(nz: int) -> np.ndarray:
    k = np.arange(nz, dtype=np.float64)
    return np.minimum(20.0 * 1.1 ** k, 500.0)


def _terrain(nx, ny, dx, n_hills, rng) -> np.ndarray:
    lx, ly = (nx - 1) * dx, (ny - 1) * dx
    xs = np.arange(nx, dtype=np.float64) * dx
    ys = np.arange(ny, dtype=np.float64) * dx
    h = np.zeros((ny, nx), dtype=np.float64)
    xc = rng.uniform(0.0, max(lx, dx), n_hills)
    yc = rng.uniform(0.0, max(ly, dx), n_hills)
    hh = rng.uniform(200.0, 2000.0, n_hills)
    hw = rng.uniform(1000.0, 10000.0, n_hills)
    sig = hw / math.sqrt(2.0 * math.log(2.0))
    for m in range(n_hills):
        gx = np.exp(-((xs - xc[m]) ** 2) / (2.0 * sig[m] ** 2))
        gy = np.exp(-((ys - yc[m]) ** 2) / (2.0 * sig[m] ** 2))
        h += hh[m] * np.outer(gy, gx)
    return h.astype(F32)


def build_domain(nx: int, ny: int, nz: int, dx: float = 250.0, n_hills: int = 20,
                 seed: int = 0, adv_den: bool = True, terrain: np.ndarray | None = None,
                 dz_levels: np.ndarray | None = None) -> Domain:
    """Terrain + Gal-Chen metrics, restating domain_obj.F90:1933-2056 and 2195-2265."""
    rng = np.random.default_rng(seed)
    dx = F32(dx)
    if terrain is None:
        terrain = _terrain(nx, ny, float(dx), n_hills, rng) if n_hills > 0 else np.zeros((ny, nx), F32)
    terrain = np.ascontiguousarray(terrain, dtype=F32)
    if dz_levels is None:
        nom = nominal_levels(nz)
        scale = (float(terrain.max()) + nom.sum()) / nom.sum()
        dz_levels = (nom * scale).astype(F32)
    dz = np.ascontiguousarray(dz_levels, dtype=F32)
    # smooth_height = sum(dz(1:max_level))  (sequential FP32 sum)
    H = F32(0.0)
    for k in range(nz):
        H = F32(H + dz[k])
    jac2 = ((H - terrain) / H).astype(F32)                      # (:1982-1983)
    jac = np.repeat(jac2[:, None, :], nz, axis=1)                # jacobian(:,k,:) = jacobian(:,k-1,:)
    dz_int = (dz[None, :, None] * jac).astype(F32)               # dz_interface = dz(k)*jacobian
    # mass-level heights z (:1985-2001)
    z = np.empty_like(jac)
    z[:, 0, :] = terrain + (dz[0] / F32(2)) * jac[:, 0, :]
    for k in range(1, nz):
        z[:, k, :] = z[:, k - 1, :] + ((dz[k] / F32(2)) * jac[:, k, :] + (dz[k - 1] / F32(2)) * jac[:, k - 1, :])
    # jacobian_u / jacobian_v (:2008-2020), neighbour jacobian == jacobian at one rank
    ju = np.empty((ny, nz, nx + 1), F32)
    ju[:, :, 0] = jac[:, :, 0]
    ju[:, :, nx] = jac[:, :, nx - 1]
    ju[:, :, 1:nx] = (jac[:, :, 1:nx] + jac[:, :, 0:nx - 1]) / F32(2)
    jv = np.empty((ny + 1, nz, nx), F32)
    jv[0] = jac[0]
    jv[ny] = jac[ny - 1]
    jv[1:ny] = (jac[1:ny] + jac[0:ny - 1]) / F32(2)
    # jacobian_w (:2022-2026)
    jw = np.empty_like(jac)
    jw[:, nz - 1, :] = F32(1.0)
    jw[:, :nz - 1, :] = (dz_int[:, 1:, :] * jac[:, :nz - 1, :] + dz_int[:, :nz - 1, :] * jac[:, 1:, :]) / \
                        (dz_int[:, :nz - 1, :] + dz_int[:, 1:, :])
    # setup_dzdxy (:2195-2265)
    nzh = np.empty_like(jac)
    nzh[:, 0, :] = terrain + (dz[0] / F32(2)) * jac[:, 0, :]
    for k in range(1, nz):
        nzh[:, k, :] = nzh[:, k - 1, :] + ((dz[k] / F32(2)) * jac[:, k, :]) + ((dz[k - 1] / F32(2)) * jac[:, k - 1, :])
    two_dx = F32(2) * dx
    dzdx = np.zeros_like(jac)
    dzdx[:, :, 1:nx - 1] = (nzh[:, :, 2:nx] - nzh[:, :, 0:nx - 2]) / two_dx
    dzdx[:, :, 0] = (F32(-3) * nzh[:, :, 0] + F32(4) * nzh[:, :, 1] - nzh[:, :, 2]) / two_dx
    dzdx[:, :, nx - 1] = (F32(3) * nzh[:, :, nx - 1] - F32(4) * nzh[:, :, nx - 2] + nzh[:, :, nx - 3]) / two_dx
    dzdx_u = np.empty((ny, nz, nx + 1), F32)
    dzdx_u[:, :, 1:nx] = (nzh[:, :, 1:nx] - nzh[:, :, 0:nx - 1]) / dx
    dzdx_u[:, :, 0] = dzdx[:, :, 0] * F32(1.5) - dzdx[:, :, 1] * F32(0.5)
    dzdx_u[:, :, nx] = dzdx[:, :, nx - 1] * F32(1.5) - dzdx[:, :, nx - 2] * F32(0.5)
    dzdy = np.zeros_like(jac)
    dzdy[1:ny - 1] = (nzh[2:ny] - nzh[0:ny - 2]) / two_dx
    dzdy[0] = (F32(-3) * nzh[0] + F32(4) * nzh[1] - nzh[2]) / two_dx
    dzdy[ny - 1] = (F32(3) * nzh[ny - 1] - F32(4) * nzh[ny - 2] + nzh[ny - 3]) / two_dx
    dzdy_v = np.empty((ny + 1, nz, nx), F32)
    dzdy_v[1:ny] = (nzh[1:ny] - nzh[0:ny - 1]) / dx
    dzdy_v[0] = dzdy[0] * F32(1.5) - dzdy[1] * F32(0.5)
    dzdy_v[ny] = dzdy[ny - 1] * F32(1.5) - dzdy[ny - 2] * F32(0.5)
    adz = np.ascontiguousarray(np.broadcast_to(dz[None, :, None], (ny, nz, nx)), dtype=F32)
    if adv_den:
        density = (F32(1.2) * np.exp(-z.astype(np.float64) / 8000.0)).astype(F32)
    else:
        density = np.ones_like(jac)
    one = lambda *s: np.ones(s, F32)  # noqa: E731
    c = np.ascontiguousarray
    return Domain(nx=nx, ny=ny, nz=nz, dx=float(dx), terrain=terrain, dz_levels=dz,
                  jacobian=c(jac), jacobian_u=ju, jacobian_v=jv, jacobian_w=c(jw),
                  dzdx=c(dzdx), dzdy=c(dzdy), dzdx_u=dzdx_u, dzdy_v=dzdy_v,
                  advection_dz=adz, neighbor_terrain=terrain.copy(), density=c(density), z=c(z),
                  mapfac_mx_u=one(ny, nx + 1), mapfac_my_v=one(ny + 1, nx),
                  mapfac_my_u=one(ny, nx + 1), mapfac_mx_v=one(ny + 1, nx), mapfac_mxy=one(ny, nx),
                  seed=seed)


def _face_agl(d: Domain, axis: str) -> np.ndarray:
    agl = (d.z - d.terrain[:, None, :]).astype(np.float64)
    if axis == "u":
        out = np.empty((d.ny, d.nz, d.nx + 1))
        out[:, :, 1:d.nx] = 0.5 * (agl[:, :, 1:] + agl[:, :, :-1])
        out[:, :, 0] = agl[:, :, 0]
        out[:, :, d.nx] = agl[:, :, d.nx - 1]
    else:
        out = np.empty((d.ny + 1, d.nz, d.nx))
        out[1:d.ny] = 0.5 * (agl[1:] + agl[:-1])
        out[0] = agl[0]
        out[d.ny] = agl[d.ny - 1]
    return out


def smooth_alpha(d: Domain, rng, lo: float = 0.3, hi: float = 1.0, n_modes: int = 8) -> np.ndarray:
    """Smooth seeded stability field mapped affinely onto [lo, hi]."""
    x = np.arange(d.nx, dtype=np.float64)[None, None, :] / max(d.nx, 1)
    y = np.arange(d.ny, dtype=np.float64)[:, None, None] / max(d.ny, 1)
    zz = np.arange(d.nz, dtype=np.float64)[None, :, None] / max(d.nz, 1)
    f = np.zeros((d.ny, d.nz, d.nx), dtype=np.float64)
    for _ in range(n_modes):
        kx, ky = rng.integers(1, 4, 2)
        ph = rng.uniform(0, 2 * math.pi)
        amp = rng.normal()
        decay = rng.uniform(0.5, 3.0)
        f += amp * np.cos(2 * math.pi * (kx * x + ky * y) + ph) * np.exp(-decay * zz)
    f = (f - f.min()) / max(f.max() - f.min(), 1e-12)
    return (lo + (hi - lo) * f).astype(F32)


def build_case(nx: int, ny: int, nz: int, dx: float = 250.0, n_hills: int = 20, seed: int = 0,
               adv_den: bool = True, alpha: str = "const", name: str = "") -> Case:
    d = build_domain(nx, ny, nz, dx, n_hills, seed, adv_den)
    rng = np.random.default_rng(seed + 7919)
    speed = rng.uniform(5.0, 15.0)
    theta = rng.uniform(0.0, 2.0 * math.pi)
    z0, zref = 0.1, 100.0
    prof = lambda agl: speed * np.log(np.maximum(agl, 2 * z0) / z0) / math.log(zref / z0)  # noqa: E731
    u = (prof(_face_agl(d, "u")) * math.cos(theta) + rng.standard_normal((ny, nz, nx + 1))).astype(F32)
    v = (prof(_face_agl(d, "v")) * math.sin(theta) + rng.standard_normal((ny + 1, nz, nx))).astype(F32)
    w = np.zeros((ny, nz, nx), F32)
    if alpha == "const":
        a = np.ones((ny, nz, nx), F32)
    else:
        a = smooth_alpha(d, rng)
    return Case(domain=d, u=u, v=v, w=w, alpha=a, adv_den=adv_den, name=name)


def stability_inputs(case: Case, seed: int = 0, nsect: int = 72):
    """Inputs of update_stability beside the winds: the potential temperature
    (ny, nz, nx), a stable profile 288 K + 4 K/km with N(0, 0.2) K noise, and the
    blocking heights per wind-direction sector (nsect, ny, nz, nx): U[0, 3000] m,
    the range that HICAR's terrain search (compute_terrain_blocking_heights,
    wind.F90:1571-1729) produces on these terrains, kept at least the level's
    thickness."""
    d = case.domain
    rng = np.random.default_rng(seed + 4243)
    theta = (288.0 + 0.004 * d.z.astype(np.float64) + rng.normal(0.0, 0.2, d.z.shape)).astype(F32)
    ft = rng.uniform(0.0, 3000.0, (nsect, d.ny, d.nz, d.nx))
    dz = (d.dz_levels[None, None, :, None] * d.jacobian[None]).astype(np.float64)
    ft = np.maximum(ft, dz).astype(F32)
    return theta, ft


# Workloads named by what they are (sizes from the reference's benchmark plan).
WORKLOADS = {
    "cpu64": dict(nx=64, ny=64, nz=20, n_hills=20, alpha="const"),
    "plain512": dict(nx=512, ny=512, nz=48, n_hills=20, alpha="const"),
    "mixed1024": dict(nx=1024, ny=1024, nz=64, n_hills=60, alpha="smooth"),
    "train128": dict(nx=128, ny=128, nz=32, n_hills=20, alpha="const"),
}


def unit_test_case(nx: int = 64, ny: int = 64, nz: int = 20) -> Case:
    """The reference unit test's set-up (tests/unit/test_wind_iterative.F90:68-87,179-207):
    flat plane, dx = 250 m, alpha = 1, density = 1, u = 8 cos(2 pi (i-ids)/Lx),
    v = 6 sin(2 pi (j-jds)/Ly), w = 0."""
    d = build_domain(nx, ny, nz, 250.0, 0, 0, adv_den=False, terrain=np.zeros((ny, nx), F32),
                     dz_levels=nominal_levels(nz).astype(F32))
    lx = F32(max(nx - 1, 1))
    ly = F32(max(ny - 1, 1))
    pi = F32(math.pi)
    ii = np.arange(1, nx + 2, dtype=F32)
    jj = np.arange(1, ny + 2, dtype=F32)
    u1 = (F32(8.0) * np.cos(F32(2.0) * pi * (ii - F32(1)) / lx)).astype(F32)
    v1 = (F32(6.0) * np.sin(F32(2.0) * pi * (jj - F32(1)) / ly)).astype(F32)
    u = np.ascontiguousarray(np.broadcast_to(u1[None, None, :], (ny, nz, nx + 1)), dtype=F32)
    v = np.ascontiguousarray(np.broadcast_to(v1[:, None, None], (ny + 1, nz, nx)), dtype=F32)
    w = np.zeros((ny, nz, nx), F32)
    a = np.ones((ny, nz, nx), F32)
    return Case(domain=d, u=u, v=v, w=w, alpha=a, adv_den=False, name="unit_test")
