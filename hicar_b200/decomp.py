"""Decomposed wind solves over several ranks: HICAR's 2-D x-y block
decomposition (grid_obj.F90:340-364) with one-cell halos and the multi-rank
BiCGStab of wind_iterative.F90:555-791 -- the Krylov halo exchange of p^ and s^
before each operator apply (exchange_krylov_halos, :1552-1733) and the FP64
allreduces of the 3 set-up, the 1 sigma and the 5 packed dot products
(:604-729).  The preconditioner keeps a zero halo (:1262-1266).

The library computes (hicarw_dist_* in include/hicarw.h), the host
communicates.  `rank_schedule` is the reference's iteration as a generator that
yields at every communication point; a driver performs the communication:

* `run_distributed`: torch.distributed point-to-point face exchange and
  all_reduce (NCCL between GPUs, or gloo on the host), one process per rank;
* `run_local`: every rank's generator in one process, the exchange done by
  copies and the allreduce by a sum -- for testing the schedule on one device.

A rank is any object with the primitives of `CudaRank` (the library); the CPU
test suite drives a numpy restatement of the same primitives through gloo.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

from . import _capi

WEST, EAST, SOUTH, NORTH = 0, 1, 2, 3
OPPOSITE = {WEST: EAST, EAST: WEST, SOUTH: NORTH, NORTH: SOUTH}


@dataclasses.dataclass
class Decomposition:
    """px x py blocks of an nx x ny grid (ranks x-fastest, as HICAR's images)."""
    nx: int
    ny: int
    px: int
    py: int

    @property
    def size(self) -> int:
        return self.px * self.py

    def coords(self, rank: int):
        return rank % self.px, rank // self.px

    @staticmethod
    def _split(n, p, q):
        base, extra = divmod(n, p)
        lo = q * base + min(q, extra) + 1
        return lo, lo + base + (1 if q < extra else 0) - 1

    def block(self, rank: int):
        """(i0, i1, j0, j1): the rank's interior cells, 1-based inclusive."""
        cx, cy = self.coords(rank)
        return self._split(self.nx, self.px, cx) + self._split(self.ny, self.py, cy)

    def neighbors(self, rank: int) -> dict:
        """side -> neighbouring rank, for the sides that border another rank."""
        cx, cy = self.coords(rank)
        out = {}
        if cx > 0:
            out[WEST] = rank - 1
        if cx < self.px - 1:
            out[EAST] = rank + 1
        if cy > 0:
            out[SOUTH] = rank - self.px
        if cy < self.py - 1:
            out[NORTH] = rank + self.px
        return out

    def edges(self, rank: int) -> int:
        """Rank-edge bits of hicarw_dist_configure (1 W, 2 E, 4 S, 8 N)."""
        return sum(1 << s for s in self.neighbors(rank))

    def local(self, rank: int, a):
        """The rank's block with its one-cell ring out of a global (ny+2, nz+2, nx+2) array."""
        i0, i1, j0, j1 = self.block(rank)
        return a[j0 - 1:j1 + 2, :, i0 - 1:i1 + 2]

    def interior(self, rank: int, a):
        """The rank's interior cells out of a global (ny, nz, nx) cell array (any leading axes)."""
        i0, i1, j0, j1 = self.block(rank)
        return a[..., j0 - 1:j1, :, i0 - 1:i1]


def face_shape(nx: int, ny: int, nz: int, side: int):
    return (ny + 2, nz + 2) if side in (WEST, EAST) else (nz + 2, nx + 2)


def rank_schedule(rank_solver, neighbors: dict, rhs, max_iters: int):
    """One rank's BiCGStab (reference schedule) as a generator.  Yields
    ("allreduce", buf) -- buf summed over ranks in place before resuming -- and
    ("exchange", sends, recvs) -- sends[side] to the neighbour on that side,
    recvs[side] from it -- at the reference's communication points.  Returns
    the solve statistics."""
    r = rank_solver
    t3 = r.setup(rhs)
    yield ("allreduce", t3)
    r.apply(0, t3)
    for _ in range(max_iters + 1):
        if r.stopped():
            break
        for which in (0, 1):
            r.precond(which)
            sends, recvs = {}, {}
            for side in neighbors:
                sends[side] = r.face(which, side, unpack=False)
                recvs[side] = r.face_buffer(side)
            yield ("exchange", sends, recvs)
            for side, buf in recvs.items():
                r.face(which, side, unpack=True, buf=buf)
            tot = r.spmv(which)
            yield ("allreduce", tot)
            r.apply(1 + which, tot)
        r.update()
    return r.stats()


def run_local(schedules, decomposition: Decomposition):
    """Drive every rank's schedule in one process: at each communication point
    all ranks have yielded the same operation; allreduce = the sum over ranks
    copied back to each, exchange = copies of the neighbours' faces."""
    ops = [next(g) for g in schedules]
    results = [None] * len(schedules)
    while True:
        kinds = {op[0] for op in ops if op is not None}
        if not kinds:
            return results
        assert len(kinds) == 1, kinds
        if "allreduce" in kinds:
            total = sum(op[1] for op in ops)
            for op in ops:
                op[1].copy_(total)
        else:
            for rank, op in enumerate(ops):
                for side, buf in op[2].items():
                    nbr = decomposition.neighbors(rank)[side]
                    buf.copy_(ops[nbr][1][OPPOSITE[side]])
        nxt = []
        for q, g in enumerate(schedules):
            try:
                nxt.append(g.send(None))
            except StopIteration as e:
                results[q] = e.value
                nxt.append(None)
        ops = nxt


def run_distributed(schedule, decomposition: Decomposition, rank: int, dist):
    """Drive this rank's schedule with torch.distributed (NCCL for device
    buffers, gloo for host ones): batched isend/irecv of the faces, all_reduce
    of the totals.  Every rank takes the same collective steps in the same order."""
    nbrs = decomposition.neighbors(rank)
    try:
        op = next(schedule)
        while True:
            if op[0] == "allreduce":
                dist.all_reduce(op[1], op=dist.ReduceOp.SUM)
            else:
                p2p = []
                for side, nbr in nbrs.items():
                    p2p.append(dist.P2POp(dist.isend, op[1][side], nbr))
                    p2p.append(dist.P2POp(dist.irecv, op[2][side], nbr))
                if p2p:
                    for req in dist.batch_isend_irecv(p2p):
                        req.wait()
            op = schedule.send(None)
    except StopIteration as e:
        return e.value


class CudaRank:
    """One rank's block on this GPU: a library handle of the block's size with
    the block's probed coefficients, its rank edges marked; the primitives of
    rank_schedule on device buffers."""

    def __init__(self, dom, coefs, edges: int, options=None, stream=None):
        import torch

        from . import wind_iterative as wi
        from .domain import ptr
        self.torch = torch
        self.lib = _capi.load()
        self.dom = dom
        self.s = C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        opt = options or wi.WindOptions()
        g = _capi.Grid(dom.nx, dom.ny, dom.nz, dom.dx, 1)
        m = _capi.Metrics(*[ptr(dom.metrics[n]) for n in _capi.METRIC_FIELDS])
        h = C.c_void_p()
        _capi.check(self.lib.hicarw_init_iter_winds(C.byref(g), C.byref(opt.to_c()), C.byref(m), _capi.MEM_DEVICE,
                                                    self.s, C.byref(h)))
        self.h = h
        coefs = torch.as_tensor(coefs, dtype=torch.float32).contiguous().cuda()
        _capi.check(self.lib.hicarw_set_coefs(h, coefs.data_ptr(), 1, _capi.MEM_DEVICE, self.s), h)
        _capi.check(self.lib.hicarw_dist_configure(h, edges), h)
        self.faces = {}

    def _tot(self, n):
        return self.torch.zeros(n, dtype=self.torch.float64, device="cuda")

    def setup(self, rhs):
        t = self._tot(3)
        self.rhs = self.torch.as_tensor(rhs, dtype=self.torch.float64).contiguous().cuda()
        _capi.check(self.lib.hicarw_dist_setup(self.h, self.rhs.data_ptr(), t.data_ptr(), _capi.MEM_DEVICE, self.s),
                    self.h)
        return t

    def apply(self, kind, tot):
        _capi.check(self.lib.hicarw_dist_apply(self.h, kind, tot.data_ptr(), _capi.MEM_DEVICE, self.s), self.h)

    def precond(self, which):
        _capi.check(self.lib.hicarw_dist_precond(self.h, which, self.s), self.h)

    def face_buffer(self, side):
        return self.torch.empty(face_shape(self.dom.nx, self.dom.ny, self.dom.nz, side), dtype=self.torch.float64,
                                device="cuda")

    def face(self, vec, side, unpack, buf=None):
        if buf is None:
            buf = self.face_buffer(side)
        _capi.check(self.lib.hicarw_dist_face(self.h, vec, side, buf.data_ptr(), int(unpack), self.s), self.h)
        return buf

    def spmv(self, which):
        t = self._tot(1 if which == 0 else 5)
        _capi.check(self.lib.hicarw_dist_spmv(self.h, which, t.data_ptr(), _capi.MEM_DEVICE, self.s), self.h)
        return t

    def update(self):
        _capi.check(self.lib.hicarw_dist_update(self.h, self.s), self.h)

    def stopped(self) -> bool:
        stop = C.c_int()
        _capi.check(self.lib.hicarw_dist_state(self.h, C.byref(stop), None, self.s), self.h)
        return bool(stop.value)

    def stats(self) -> dict:
        st = _capi.Stats()
        _capi.check(self.lib.hicarw_dist_state(self.h, None, C.byref(st), self.s), self.h)
        return st.as_dict()

    def lam(self):
        d = self.dom
        out = self.torch.empty((d.ny + 2, d.nz + 2, d.nx + 2), dtype=self.torch.float64, device="cuda")
        _capi.check(self.lib.hicarw_get_lambda(self.h, out.data_ptr(), _capi.MEM_DEVICE, self.s), self.h)
        return out

    def close(self):
        if self.h:
            self.lib.hicarw_finalize_iter_winds(self.h)
            self.h = None


def local_case(case, dec: Decomposition, rank: int):
    """The rank's block of a global case (metrics, density, winds, alpha) as a
    case of the block's size: cell arrays sliced, face arrays with their
    staggered extra column or row."""
    import copy

    import numpy as np
    i0, i1, j0, j1 = dec.block(rank)
    d = case.domain
    sl_c = (slice(j0 - 1, j1), slice(None), slice(i0 - 1, i1))
    sl_u = (slice(j0 - 1, j1), slice(None), slice(i0 - 1, i1 + 1))
    sl_v = (slice(j0 - 1, j1 + 1), slice(None), slice(i0 - 1, i1))
    nd = copy.copy(d)
    nd.nx, nd.ny = i1 - i0 + 1, j1 - j0 + 1
    for name in ("jacobian", "jacobian_w", "dzdx", "dzdy", "advection_dz", "density", "z"):
        setattr(nd, name, np.ascontiguousarray(getattr(d, name)[sl_c]))
    for name in ("jacobian_u", "dzdx_u"):
        setattr(nd, name, np.ascontiguousarray(getattr(d, name)[sl_u]))
    for name in ("jacobian_v", "dzdy_v"):
        setattr(nd, name, np.ascontiguousarray(getattr(d, name)[sl_v]))
    nd.terrain = np.ascontiguousarray(d.terrain[j0 - 1:j1, i0 - 1:i1])
    nd.neighbor_terrain = np.ascontiguousarray(d.neighbor_terrain[j0 - 1:j1, i0 - 1:i1])
    nd.mapfac_mxy = np.ascontiguousarray(d.mapfac_mxy[j0 - 1:j1, i0 - 1:i1])
    for name in ("mapfac_mx_u", "mapfac_my_u"):
        setattr(nd, name, np.ascontiguousarray(getattr(d, name)[j0 - 1:j1, i0 - 1:i1 + 1]))
    for name in ("mapfac_my_v", "mapfac_mx_v"):
        setattr(nd, name, np.ascontiguousarray(getattr(d, name)[j0 - 1:j1 + 1, i0 - 1:i1]))
    nc = copy.copy(case)
    nc.domain = nd
    nc.u = np.ascontiguousarray(case.u[sl_u])
    nc.v = np.ascontiguousarray(case.v[sl_v])
    nc.w = np.ascontiguousarray(case.w[sl_c])
    nc.alpha = np.ascontiguousarray(case.alpha[sl_c])
    return nc
