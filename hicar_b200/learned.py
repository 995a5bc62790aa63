"""Learned preconditioner for the wind solver: host side of the tensor-core
convolutions and the 3-level U-Net (hicar_b200/csrc/k_conv.cu, k_unet.cu).

Activation tensors live in the library's "act layout" (BF16, channel groups of
8, zero halo): `to_act` / `from_act` convert (C, ny, nz, nx) float tensors to
and from it.  Convolution weights are FP32 [27][cin][cout] with tap
t = (dj+1)*9 + (dk+1)*3 + (di+1)."""
from __future__ import annotations

import ctypes as C

from . import _capi


def _torch():
    import torch
    return torch


def act_pitch(nx: int) -> int:
    return ((nx + 127) // 128) * 128 + 2


def act_empty(nx: int, ny: int, nz: int, ch: int, device="cuda"):
    """Zeroed act-layout tensor, shape (ny+2, nz+2, ch/8, PX, 8), BF16."""
    torch = _torch()
    if ch % 8:
        raise ValueError("channel count must be a multiple of 8")
    return torch.zeros((ny + 2, nz + 2, ch // 8, act_pitch(nx), 8), dtype=torch.bfloat16, device=device)


def to_act(x, device="cuda"):
    """(C, ny, nz, nx) float tensor -> act-layout BF16 tensor."""
    torch = _torch()
    ch, ny, nz, nx = x.shape
    out = act_empty(nx, ny, nz, ch, device)
    out[1:ny + 1, 1:nz + 1, :, 1:nx + 1, :] = (
        x.to(device=device, dtype=torch.float32).reshape(ch // 8, 8, ny, nz, nx).permute(2, 3, 0, 4, 1)
        .to(torch.bfloat16))
    return out


def from_act(a, nx: int):
    """act-layout tensor -> (C, ny, nz, nx) float32 tensor (same device)."""
    torch = _torch()
    ny, nz, g = a.shape[0] - 2, a.shape[1] - 2, a.shape[2]
    v = a[1:ny + 1, 1:nz + 1, :, 1:nx + 1, :].to(torch.float32)  # (ny, nz, G, nx, 8)
    return v.permute(2, 4, 0, 1, 3).reshape(g * 8, ny, nz, nx).contiguous()


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def conv3(x_act, w, bias, nx, ny, nz, cin, cout, *, skip=None, mask=None, relu=False, transpose=False,
          want_out=True, want_out0=False, stream=None):
    """One tensor-core 3x3x3 convolution (transpose=True: its data-gradient form,
    cout -> cin channels).  Returns (out_act or None, out0 or None)."""
    torch = _torch()
    co = cin if transpose else cout
    out = act_empty(nx, ny, nz, co, x_act.device) if want_out else None
    out0 = torch.empty((ny, nz, nx), dtype=torch.float32, device=x_act.device) if want_out0 else None
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = _capi.load().hicarw_nn_conv3(cin, cout, nx, ny, nz, _ptr(x_act), _ptr(w), _ptr(bias), _ptr(skip),
                                      _ptr(mask), int(relu), int(transpose), _ptr(out), _ptr(out0), C.c_void_p(s))
    if rc != 0:
        raise RuntimeError(f"hicarw_nn_conv3 failed ({rc})")
    return out, out0


def conv3_wgrad(x_act, dy_act, nx, ny, nz, cin, cout, stream=None):
    """(dW [27][cin][cout], db [cout]) of one convolution, FP32."""
    torch = _torch()
    dw = torch.zeros((27, cin, cout), dtype=torch.float32, device=x_act.device)
    db = torch.zeros((cout,), dtype=torch.float32, device=x_act.device)
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = _capi.load().hicarw_nn_conv3_wgrad(cin, cout, nx, ny, nz, _ptr(x_act), _ptr(dy_act), _ptr(dw), _ptr(db),
                                            C.c_void_p(s))
    if rc != 0:
        raise RuntimeError(f"hicarw_nn_conv3_wgrad failed ({rc})")
    return dw, db


class UNet:
    """The learned preconditioner's network for one grid size (owns its device
    activations); parameters are an FP32 vector (conv weights [27][cin][cout]
    then bias, convs a..g)."""

    def __init__(self, nx: int, ny: int, nz: int, seed: int = 0):
        self.lib = _capi.load()
        self.nx, self.ny, self.nz = nx, ny, nz
        h = C.c_void_p()
        rc = self.lib.hicarw_unet_create(nx, ny, nz, seed, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"hicarw_unet_create failed ({rc})")
        self.h = h

    def close(self):
        if self.h:
            self.lib.hicarw_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _s(stream=None):
        torch = _torch()
        return C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _check(rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc})")

    @property
    def nparams(self) -> int:
        return int(self.lib.hicarw_unet_num_params(self.h))

    def params(self):
        torch = _torch()
        p = torch.empty(self.nparams, dtype=torch.float32, device="cuda")
        self._check(self.lib.hicarw_unet_get_params(self.h, _ptr(p), _capi.MEM_DEVICE, self._s()), "get_params")
        return p

    def set_params(self, p):
        torch = _torch()
        p = p.to(device="cuda", dtype=torch.float32).contiguous()
        self._check(self.lib.hicarw_unet_set_params(self.h, _ptr(p), _capi.MEM_DEVICE, self._s()), "set_params")

    def grads(self):
        torch = _torch()
        g = torch.empty(self.nparams, dtype=torch.float32, device="cuda")
        self._check(self.lib.hicarw_unet_get_grads(self.h, _ptr(g), _capi.MEM_DEVICE, self._s()), "get_grads")
        return g

    def zero_grads(self):
        self._check(self.lib.hicarw_unet_zero_grads(self.h, self._s()), "zero_grads")

    def features(self, handle, r):
        """(x0 act tensor, rms) of residual r (cuda FP64 (ny+2, nz+2, nx+2))."""
        x0 = act_empty(self.nx, self.ny, self.nz, 16, "cuda")
        rms = C.c_float()
        self._check(self.lib.hicarw_unet_features(self.h, handle, _ptr(r), _ptr(x0), C.byref(rms), self._s()),
                    "features")
        return x0, rms.value

    def forward(self, x0):
        torch = _torch()
        o = torch.empty((self.ny, self.nz, self.nx), dtype=torch.float32, device="cuda")
        self._check(self.lib.hicarw_unet_forward(self.h, _ptr(x0), _ptr(o), self._s()), "forward")
        return o

    def backward(self, target, weight: float = 1.0) -> float:
        """loss = weight * mean((O_0 - target)^2); its gradients are accumulated."""
        loss = C.c_float()
        self._check(self.lib.hicarw_unet_backward(self.h, _ptr(target), C.c_float(weight), C.byref(loss), self._s()),
                    "backward")
        return loss.value

    def backward_residual(self, coefs, rhat, weight: float = 1.0) -> float:
        """loss = weight * mean((A z - rhat)^2), z = O_0 / coef_A; gradients accumulated."""
        loss = C.c_float()
        self._check(self.lib.hicarw_unet_backward_residual(self.h, _ptr(coefs), _ptr(rhat), C.c_float(weight),
                                                           C.byref(loss), self._s()), "backward_residual")
        return loss.value

    def adam_step(self, lr: float):
        self._check(self.lib.hicarw_unet_adam_step(self.h, C.c_float(lr), self._s()), "adam_step")

    def apply(self, handle, r):
        torch = _torch()
        z = torch.zeros_like(r)
        self._check(self.lib.hicarw_unet_apply(self.h, handle, _ptr(r), _ptr(z), self._s()), "apply")
        return z

    def attach(self, handle):
        """Use this network for HICARW_PRECOND_LEARNED solves of `handle` (same grid)."""
        self._check(self.lib.hicarw_set_learned_precond(handle, self.h), "set_learned_precond")


def random_residual(nx, ny, nz, gen, device="cuda"):
    """A residual-like field (FP64, (ny+2, nz+2, nx+2), zero ghost cells): white
    noise smoothed by a random number of 3x3 x-y box passes (0..16) and z passes
    (0..2), so that the training set spans rough and smooth components."""
    torch = _torch()
    F = torch.nn.functional
    x = torch.randn((1, 1, ny, nz, nx), generator=gen, dtype=torch.float64).to(device)
    nxy = int(torch.randint(0, 17, (1,), generator=gen))
    nzp = int(torch.randint(0, 3, (1,), generator=gen))
    for _ in range(nxy):
        x = F.avg_pool3d(F.pad(x, (1, 1, 0, 0, 1, 1), mode="replicate"), (3, 1, 3), stride=1)
    for _ in range(nzp):
        x = F.avg_pool3d(F.pad(x, (0, 0, 1, 1, 0, 0), mode="replicate"), (1, 3, 1), stride=1)
    x = x / x.std()
    r = torch.zeros((ny + 2, nz + 2, nx + 2), dtype=torch.float64, device=device)
    r[1:-1, 1:-1, 1:-1] = x[0, 0]
    return r


def calibrated_handle(case):
    """(DeviceDomain, handle) with the case's probed operator, calibrated as in update_winds."""
    torch = _torch()
    from . import wind, wind_iterative as wi
    from .domain import DeviceDomain
    dom = DeviceDomain.from_case(case, "cuda")
    opt = wi.WindOptions(tol_rel=1e-6)
    wi.init_iter_winds(dom, opt)
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    wind.update_winds_iterative(dom, opt, div)
    return dom, wi.handle(dom.nest_indx)


def probed_handle(case):
    """(DeviceDomain, handle) with the case's probed operator from the 27-colour
    calibration alone (no solves before it): the operator is the same as
    after update_winds' first update, which calibrates with the same alpha."""
    from . import wind, wind_iterative as wi
    from .domain import DeviceDomain
    dom = DeviceDomain.from_case(case, "cuda")
    opt = wi.WindOptions(tol_rel=1e-6)
    wi.init_iter_winds(dom, opt)
    wind.calibrate_projection_operator(dom, opt)
    return dom, wi.handle(dom.nest_indx)


SOLVER_ITERS = (1, 3, 8, 16, 32, 64, 128, 256)  # plain-solver iterations whose residuals are logged


def training_pairs(case, net: UNet, n_samples: int, seed: int = 0, solve: bool = False, tol: float = 1e-8,
                   source: str = "random"):
    """Training samples of one terrain case: the network input features x0 of a
    residual r, the unit-rms residual rhat = r / rms(r) (FP32, (ny, nz, nx)) and the
    operator's FP32 coefficients (15, ny, nz, nx), which the residual loss
    ||A z - rhat||^2 needs.  source="random": r from random_residual;
    source="solver": r = b - A x_k, the residual after k = SOLVER_ITERS[(q + seed) % 8] iterations
    of the plain (Jacobi-preconditioned) BiCGStab on the case's own right-hand
    side b = -2 div(u, v, w), i.e. the residuals the solver itself produces.  With
    solve=True also the exact step e = A^-1 r (FGMRES + multigrid to `tol`) as the
    target e * coef_A / rms(r) of the supervised loss.  Each sample is
    (x0, rhat, coefs, target or None).  The handles made here are released again."""
    torch = _torch()
    from . import wind, wind_iterative as wi
    dom, h = calibrated_handle(case)
    lib = _capi.load()
    exact = wi.WindOptions(tol_rel=tol, wind_solver_iterations=2000, solver=_capi.SOLVER_FGMRES,
                           precond=_capi.PRECOND_MG)
    wi.set_options(exact)
    coefs = torch.empty((15, dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    _capi.check(lib.hicarw_get_coefs(h, _ptr(coefs), _capi.MEM_DEVICE, None), h)
    diag = coefs[0].double()
    gen = torch.Generator().manual_seed(seed)
    b = None
    if source == "solver":
        div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
        dom.set_winds(case.u, case.v, case.w)
        wind.calc_divergence(div, dom, use_dqdt=True)
        b = torch.zeros((dom.ny + 2, dom.nz + 2, dom.nx + 2), dtype=torch.float64, device="cuda")
        b[1:-1, 1:-1, 1:-1] = -2.0 * div.double()  # compute_rhs_3d (wind_iterative.F90:1513-1530)
    out = []
    st = _capi.Stats()
    for q in range(n_samples):
        if source == "solver":
            k = SOLVER_ITERS[(q + seed) % len(SOLVER_ITERS)]
            wi.set_options(wi.WindOptions(tol_rel=1e-30, tol_abs=0.0, wind_solver_iterations=k))
            lib.hicarw_reset_solution(h, None)
            _capi.check(lib.hicarw_solve_rhs(h, _ptr(b), _capi.MEM_DEVICE, None, C.byref(st)), h)
            xk = torch.empty_like(b)
            _capi.check(lib.hicarw_get_lambda(h, _ptr(xk), _capi.MEM_DEVICE, None), h)
            ax = torch.empty_like(b)
            _capi.check(lib.hicarw_apply_operator(h, _ptr(xk), _ptr(ax), _capi.MEM_DEVICE, None), h)
            r = b - ax
            r[0], r[-1], r[:, 0], r[:, -1], r[:, :, 0], r[:, :, -1] = 0, 0, 0, 0, 0, 0
            wi.set_options(exact)
        else:
            r = random_residual(dom.nx, dom.ny, dom.nz, gen)
        x0, rms = net.features(h, r)
        rhat = (r[1:-1, 1:-1, 1:-1] / rms).float().contiguous()
        target = None
        if solve:
            lib.hicarw_reset_solution(h, None)
            _capi.check(lib.hicarw_solve_rhs(h, _ptr(r), _capi.MEM_DEVICE, None, C.byref(st)), h)
            e = torch.empty_like(r)
            _capi.check(lib.hicarw_get_lambda(h, _ptr(e), _capi.MEM_DEVICE, None), h)
            target = (e[1:-1, 1:-1, 1:-1] * diag / rms).float().contiguous()
        out.append((x0, rhat, coefs, target))
    wi.finalize_iter_winds()
    wind.reset()
    return out


# The V-cycle of the composite preconditioner (V(0,1) on the finest level, omega 1,
# W-cycles on levels 2-4): the cycle the benchmark's multigrid solves use.
MG_CYCLE = dict(mg_skip_fine_presmooth=True, mg_omega=1.0, mg_w_levels=(2, 3, 4))


def composite_pairs(case, net: UNet, ks=SOLVER_ITERS, tight_tol: float = 1e-10, cycle=None):
    """Training samples of the composite preconditioner z = M(r) + theta U(r - A M(r))
    (HICARW_PRECOND_MG_LEARNED), logged from the plain solver on one terrain:
    the case's right-hand side b = -2 div(u, v, w) is solved once tightly
    (FGMRES + V-cycle, x*), then the reference BiCGStab (Jacobi-Richardson) is
    run from x = 0, its iterate x_k logged after k = ks[0], ks[1], ...
    iterations (each leg continuing from the last iterate).  For each logged
    iterate: r = b - A x_k and e = x* - x_k, the V-cycle's z1 = M(r), and the
    pair the network learns, r' = r - A z1 and e' = e - z1 (A e' = r').  Returns
    [(x0, target)]: the network's input features of r' (act layout) and its
    supervised target e' coef_A / rms(r') (FP32 (ny, nz, nx))."""
    torch = _torch()
    from . import wind, wind_iterative as wi
    cycle = MG_CYCLE if cycle is None else cycle
    dom, h = probed_handle(case)
    lib = _capi.load()
    shape = (dom.ny + 2, dom.nz + 2, dom.nx + 2)
    coefs = torch.empty((15, dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    _capi.check(lib.hicarw_get_coefs(h, _ptr(coefs), _capi.MEM_DEVICE, None), h)
    diag = coefs[0].double()
    div = torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device="cuda")
    dom.set_winds(case.u, case.v, case.w)
    wind.calc_divergence(div, dom, use_dqdt=True)
    b = torch.zeros(shape, dtype=torch.float64, device="cuda")
    b[1:-1, 1:-1, 1:-1] = -2.0 * div.double()  # compute_rhs_3d (wind_iterative.F90:1513-1530)
    st = _capi.Stats()

    def lam():
        x = torch.empty(shape, dtype=torch.float64, device="cuda")
        _capi.check(lib.hicarw_get_lambda(h, _ptr(x), _capi.MEM_DEVICE, None), h)
        return x

    def op(x):
        y = torch.empty_like(x)
        _capi.check(lib.hicarw_apply_operator(h, _ptr(x), _ptr(y), _capi.MEM_DEVICE, None), h)
        return y

    def interior_only(a):
        a[0], a[-1], a[:, 0], a[:, -1], a[:, :, 0], a[:, :, -1] = 0, 0, 0, 0, 0, 0
        return a

    wi.set_options(wi.WindOptions(tol_rel=tight_tol, tol_abs=0.0, wind_solver_iterations=3000,
                                  solver=_capi.SOLVER_FGMRES, precond=_capi.PRECOND_MG, **cycle))
    lib.hicarw_reset_solution(h, None)
    _capi.check(lib.hicarw_solve_rhs(h, _ptr(b), _capi.MEM_DEVICE, None, C.byref(st)), h)
    xstar = lam()
    lib.hicarw_reset_solution(h, None)
    out, done = [], 0
    for k in ks:
        wi.set_options(wi.WindOptions(tol_rel=1e-30, tol_abs=0.0, wind_solver_iterations=k - done))
        _capi.check(lib.hicarw_solve_rhs(h, _ptr(b), _capi.MEM_DEVICE, None, C.byref(st)), h)
        done = k
        xk = lam()
        r = interior_only(b - op(xk))
        e = interior_only(xstar - xk)
        wi.set_options(wi.WindOptions(precond=_capi.PRECOND_MG, **cycle))
        z1 = torch.empty_like(r)
        _capi.check(lib.hicarw_apply_precond(h, _ptr(r), _ptr(z1), 0, _capi.MEM_DEVICE, None), h)
        rp = interior_only(r - op(z1))
        ep = e - z1
        x0, rms = net.features(h, rp)
        if not rms > 0.0:
            continue
        out.append((x0, (ep[1:-1, 1:-1, 1:-1] * diag / rms).float().contiguous()))
    wi.finalize_iter_winds()
    wind.reset()
    return out


def train_online(net: UNet, terrain_cases, steps_per_terrain: int = 2, batch: int = 4, lr: float = 1e-3,
                 lr_decay_every: int = 0, buffer: int = 64, seed: int = 0, log_every: int = 0,
                 time_limit_s: float = 0.0):
    """Adam on the composite's supervised loss |O_0 - T|^2 / |T|^2 (a
    relative error of the learned correction), with the samples of each
    terrain (composite_pairs) added to a replay buffer of the latest `buffer`
    samples as the terrains stream past; `steps_per_terrain` steps of `batch`
    samples drawn from the buffer follow each terrain.  `terrain_cases` yields
    seeded cases (never stored all at once).  time_limit_s > 0 stops after the
    terrain during which that much wall time has passed.  Returns the loss
    history and the number of terrains used."""
    import collections
    import time
    torch = _torch()
    t_start = time.time()
    gen = torch.Generator().manual_seed(seed)
    pool = collections.deque(maxlen=buffer)
    hist = []
    n_terrains = 0
    for case in terrain_cases:
        pool.extend(composite_pairs(case, net))
        n_terrains += 1
        if lr_decay_every and n_terrains % lr_decay_every == 0:
            lr *= 0.5
        for _ in range(steps_per_terrain):
            net.zero_grads()
            tot = 0.0
            for _ in range(batch):
                x0, target = pool[int(torch.randint(0, len(pool), (1,), generator=gen))]
                net.forward(x0)
                tot += net.backward(target, 1.0 / max(float((target.double() ** 2).mean()), 1e-30))
            net.adam_step(lr)
            hist.append(tot / batch)
        if log_every and n_terrains % log_every == 0:
            print(f"terrain {n_terrains}: loss {sum(hist[-log_every:]) / max(1, len(hist[-log_every:])):.4f} "
                  f"({time.time() - t_start:.0f} s)", flush=True)
        if time_limit_s > 0 and time.time() - t_start > time_limit_s:
            break
    return hist, n_terrains


def train(net: UNet, pairs, steps: int, lr: float = 1e-3, batch: int = 4, seed: int = 0, loss: str = "residual"):
    """Adam on the mean of the per-sample losses; returns the loss history.
    loss="residual": mean((A z - rhat)^2) with z = O_0 / coef_A, the preconditioned
    residual of a unit-rms residual, which weighs every error component by how
    much the operator amplifies it.  loss="error": ||O_0 - T||^2 / ||T||^2 against
    the exact step (pairs made with solve=True)."""
    torch = _torch()
    gen = torch.Generator().manual_seed(seed)
    hist = []
    for _ in range(steps):
        net.zero_grads()
        tot = 0.0
        for _ in range(batch):
            x0, rhat, coefs, target = pairs[int(torch.randint(0, len(pairs), (1,), generator=gen))]
            net.forward(x0)
            if loss == "residual":
                tot += net.backward_residual(coefs, rhat)
            else:
                tot += net.backward(target, 1.0 / float((target.double() ** 2).mean()))
        net.adam_step(lr)
        hist.append(tot / batch)
    return hist


def conv_benchmark(cin: int, cout: int, nx: int, ny: int, nz: int, reps: int = 5, seed: int = 0):
    """Time the tensor-core convolution (forward, bias + ReLU) on random act-layout
    data with CUDA events around `reps` launches: returns ms per launch, achieved
    TFLOP/s (54 cin cout flop per cell) and GB/s (2 (cin + cout) bytes per cell)."""
    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = act_empty(nx, ny, nz, cin)
    x[1:ny + 1, 1:nz + 1, :, 1:nx + 1, :] = torch.randn((ny, nz, cin // 8, nx, 8), generator=g, device="cuda").to(
        torch.bfloat16)
    w = torch.randn((27, cin, cout), generator=g, device="cuda") * (2.0 / (27 * cin)) ** 0.5
    b = torch.zeros(cout, device="cuda")
    out = act_empty(nx, ny, nz, cout)
    lib = _capi.load()
    s = torch.cuda.current_stream().cuda_stream

    t = C.c_float()
    rc = lib.hicarw_nn_conv3_time(cin, cout, nx, ny, nz, _ptr(x), _ptr(w), _ptr(b), _ptr(out), reps, C.c_void_p(s),
                                  C.byref(t))
    if rc != 0:
        raise RuntimeError(f"hicarw_nn_conv3_time failed ({rc})")
    ms = t.value
    cells = nx * ny * nz
    return {"cin": cin, "cout": cout, "grid": [nx, ny, nz], "ms": ms,
            "tflops": 54.0 * cin * cout * cells / (ms * 1e-3) / 1e12,
            "gbs": 2.0 * (cin + cout) * cells / (ms * 1e-3) / 1e9}


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="time the tensor-core convolution")
    ap.add_argument("--cin", type=int, default=16)
    ap.add_argument("--cout", type=int, default=16)
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nz", type=int, default=48)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    print(json.dumps(conv_benchmark(a.cin, a.cout, a.nx, a.ny, a.nz, a.reps)))


if __name__ == "__main__":
    main()
