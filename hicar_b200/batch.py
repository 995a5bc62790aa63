"""Batched wind solves of independent, unevenly sized subdomains: one calibrated
solver handle per subdomain, all solved by one CUDA graph launch
(hicarw_batch_* in include/hicarw.h) with an autotuned number of concurrent
chains and iterations per device-side loop body."""
from __future__ import annotations

import ctypes as C

from . import _capi
from .domain import DeviceDomain, ptr
from .wind_iterative import WindOptions


def _torch():
    import torch
    return torch


def subdomain_cases(n: int, seed: int = 0, nxy=(96, 512, 32), nz=(20, 48, 4), n_hills: int = 20, dx: float = 250.0):
    """n seeded subdomains with nx, ny drawn from range(*nxy) and nz from
    range(*nz), inclusive of the upper bound (the 96-subdomain batch workload:
    nx, ny in 96..512 step 32, nz in 20..48 step 4).  Yields the cases."""
    import numpy as np

    from . import cases
    rng = np.random.default_rng(seed)
    xy = np.arange(nxy[0], nxy[1] + 1, nxy[2])
    zz = np.arange(nz[0], nz[1] + 1, nz[2])
    shapes = [(int(rng.choice(xy)), int(rng.choice(xy)), int(rng.choice(zz))) for _ in range(n)]
    for i, (nx, ny, nzz) in enumerate(shapes):  # a generator: one case on the host at a time
        yield cases.build_case(nx, ny, nzz, dx, n_hills, seed=seed * 100003 + i, adv_den=True)


# Restart length of the learned subdomains' FGMRES: its basis holds 2m + 1 FP64
# vectors per subdomain, so a long restart does not fit a large batch in HBM.
LEARNED_RESTART = 10


class BatchSolver:
    """Handles for every case (created, calibrated with the 27-colour probe on the
    device) and the batch that solves them together.  learned_every = m > 0
    solves every m-th subdomain with FGMRES(LEARNED_RESTART) and the composite learned
    preconditioner (V-cycle + U-Net correction, parameters `learned_params`),
    the others with `options`."""

    def __init__(self, cases, options: WindOptions | None = None, device="cuda", stream=None,
                 learned_every: int = 0, learned_params=None):
        torch = _torch()
        self.lib = _capi.load()
        self.options = options or WindOptions(tol_rel=1e-6, wind_solver_iterations=3000,
                                              precond=_capi.PRECOND_MG, stall_iters=50)
        self.adv = bool(self.options.advect_density)
        self.stream = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self.domains, self.handles, self.divs, self.saved = [], [], [], []
        self.nets, self.learned = [], []
        self.batch = None
        try:
            for i, case in enumerate(cases):
                dom = DeviceDomain.from_case(case, device)
                g = _capi.Grid(dom.nx, dom.ny, dom.nz, dom.dx, 1)
                m = _capi.Metrics(*[ptr(dom.metrics[n]) for n in _capi.METRIC_FIELDS])
                h = C.c_void_p()
                _capi.check(self.lib.hicarw_init_iter_winds(C.byref(g), C.byref(self.options.to_c()), C.byref(m),
                                                            _capi.MEM_DEVICE, C.c_void_p(self.stream), C.byref(h)))
                self.handles.append(h)
                leak = C.c_float(0.0)
                _capi.check(self.lib.hicarw_calibrate_projection_operator(
                    h, ptr(dom.wind_alpha), ptr(dom.density) if self.adv else None, int(self.adv), ptr(dom.u_dqdt),
                    ptr(dom.v_dqdt), ptr(dom.w_dqdt), C.byref(leak), _capi.MEM_DEVICE, C.c_void_p(self.stream)), h)
                self.domains.append(dom)
                self.divs.append(torch.empty((dom.ny, dom.nz, dom.nx), dtype=torch.float32, device=device))
                self.saved.append((dom.u_dqdt.clone(), dom.v_dqdt.clone(), dom.w_dqdt.clone()))
                is_learned = learned_every > 0 and learned_params is not None and i % learned_every == learned_every - 1
                self.learned.append(is_learned)
                if is_learned:
                    from . import learned as L
                    net = L.UNet(dom.nx, dom.ny, dom.nz)
                    net.set_params(learned_params)
                    net.attach(h)
                    self.nets.append(net)
                    lo = WindOptions(**{**self.options.__dict__, "solver": _capi.SOLVER_FGMRES,
                                        "precond": _capi.PRECOND_MG_LEARNED, "fgmres_restart": LEARNED_RESTART,
                                        "stall_iters": 200, **L.MG_CYCLE})
                    _capi.check(self.lib.hicarw_set_options(h, C.byref(lo.to_c())), h)
            n = len(self.handles)
            arr = (C.c_void_p * n)(*[h.value for h in self.handles])
            b = C.c_void_p()
            _capi.check(self.lib.hicarw_batch_create(n, arr, C.byref(b)))
            self.batch = b
            self.items = (_capi.BatchItem * n)()
            for i, dom in enumerate(self.domains):
                it = self.items[i]
                it.alpha, it.div = dom.wind_alpha.data_ptr(), self.divs[i].data_ptr()
                it.density = dom.density.data_ptr() if self.adv else None
                it.u, it.v, it.w = dom.u_dqdt.data_ptr(), dom.v_dqdt.data_ptr(), dom.w_dqdt.data_ptr()
        except Exception:
            self.close()
            raise

    @property
    def n(self) -> int:
        return len(self.handles)

    @property
    def cells(self) -> int:
        return sum(d.nx * d.ny * d.nz for d in self.domains)

    def restore_winds(self):
        for dom, (u, v, w) in zip(self.domains, self.saved):
            dom.set_winds(u, v, w)

    def divergence(self):
        for h, dom, div in zip(self.handles, self.domains, self.divs):
            _capi.check(self.lib.hicarw_calc_divergence(h, ptr(dom.u_dqdt), ptr(dom.v_dqdt), ptr(dom.w_dqdt),
                                                        ptr(dom.density) if self.adv else None, ptr(div),
                                                        int(self.adv), 0, 1, _capi.MEM_DEVICE,
                                                        C.c_void_p(self.stream)), h)

    def solve(self, cold: bool = True):
        """Solve every subdomain for its current divergence and correct its winds."""
        st = (_capi.Stats * self.n)()
        _capi.check(self.lib.hicarw_batch_calc_iter_winds(self.batch, self.items, int(self.adv), int(cold),
                                                          C.c_void_p(self.stream), st))
        return [s.as_dict() for s in st]

    def step(self):
        """One batched update from the saved input winds: divergence, solve, correction."""
        self.restore_winds()
        self.divergence()
        return self.solve(cold=True)

    def configure(self, lanes: int, chunk: int):
        _capi.check(self.lib.hicarw_batch_config(self.batch, lanes, chunk))

    def config(self):
        lanes, chunk = C.c_int(), C.c_int()
        _capi.check(self.lib.hicarw_batch_get_config(self.batch, C.byref(lanes), C.byref(chunk)))
        return lanes.value, chunk.value

    def autotune(self) -> float:
        self.restore_winds()
        self.divergence()
        best = C.c_double()
        _capi.check(self.lib.hicarw_batch_autotune(self.batch, self.items, int(self.adv), C.c_void_p(self.stream),
                                                   C.byref(best)))
        return best.value

    def autotune_kernels(self, levels=(8, 16, 32, 64), feeds=(1, 0), reps: int = 2):
        """Kernel tuning per subdomain-size bucket (nz, and the column count
        nx * ny in classes of 128 x 128 columns): for the largest subdomain of
        each bucket, time `reps` solves (device solve time) with every z-march
        depth of the float4 operator kernels in `levels` and every multigrid
        post-smoother feed in `feeds` (1 tensor copies, 0 register-fed), and apply
        the fastest to the whole bucket.  Returns the table
        [{bucket, subdomains, shape, levels, feed, ms, tried}]."""
        st = _capi.Stats()
        buckets = {}
        for i, d in enumerate(self.domains):
            buckets.setdefault((d.nz, (d.nx * d.ny) // (128 * 128)), []).append(i)
        table = []
        for key in sorted(buckets):
            idx = buckets[key]
            rep = max(idx, key=lambda i: self.domains[i].nx * self.domains[i].ny)
            h, dom = self.handles[rep], self.domains[rep]
            tried = {}
            for kc in levels:
                for feed in feeds:
                    _capi.check(self.lib.hicarw_set_kernel_tuning(h, kc, feed), h)
                    ms = []
                    for _ in range(reps + 1):
                        dom.set_winds(*self.saved[rep])
                        self.lib.hicarw_reset_solution(h, C.c_void_p(self.stream))
                        _capi.check(self.lib.hicarw_calc_divergence(
                            h, ptr(dom.u_dqdt), ptr(dom.v_dqdt), ptr(dom.w_dqdt),
                            ptr(dom.density) if self.adv else None, ptr(self.divs[rep]), int(self.adv), 0, 1,
                            _capi.MEM_DEVICE, C.c_void_p(self.stream)), h)
                        _capi.check(self.lib.hicarw_calc_iter_winds(
                            h, ptr(dom.wind_alpha), ptr(self.divs[rep]), ptr(dom.density) if self.adv else None,
                            int(self.adv), ptr(dom.u_dqdt), ptr(dom.v_dqdt), ptr(dom.w_dqdt), _capi.MEM_DEVICE,
                            C.c_void_p(self.stream), C.byref(st)), h)
                        ms.append(st.solve_ms)
                    tried[f"{kc}/{feed}"] = min(ms[1:])  # the first solve captures the graphs
            best = min(tried, key=tried.get)
            kc, feed = (int(x) for x in best.split("/"))
            for i in idx:
                _capi.check(self.lib.hicarw_set_kernel_tuning(self.handles[i], kc, feed), self.handles[i])
            table.append({"bucket": {"nz": key[0], "columns_over_16384": key[1]}, "subdomains": len(idx),
                          "shape": [dom.nx, dom.ny, dom.nz], "levels": kc, "feed": feed, "ms": tried[best],
                          "tried": tried})
        self.restore_winds()
        return table

    def latencies(self):
        """Per-subdomain solve latency (ms from the batch start) of the last solve."""
        import numpy as np
        out = np.zeros(self.n)
        _capi.check(self.lib.hicarw_batch_latencies(self.batch, out.ctypes.data))
        return out

    def lambda_of(self, i: int):
        torch = _torch()
        d = self.domains[i]
        lam = torch.empty((d.ny + 2, d.nz + 2, d.nx + 2), dtype=torch.float64, device="cuda")
        _capi.check(self.lib.hicarw_get_lambda(self.handles[i], ptr(lam), _capi.MEM_DEVICE, C.c_void_p(self.stream)),
                    self.handles[i])
        return lam

    def close(self):
        if self.batch is not None:
            self.lib.hicarw_batch_destroy(self.batch)
            self.batch = None
        for h in self.handles:
            self.lib.hicarw_finalize_iter_winds(h)
        self.handles = []
        for net in self.nets:
            net.close()
        self.nets = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
