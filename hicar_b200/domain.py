"""Device-resident domain state handed to the wind solver.

HICAR keeps the model state in ``domain_t`` (src/objects/domain_h.F90); the
wind solver reads metric terms, density and alpha from it and corrects
``u%dqdt_3d``, ``v%dqdt_3d`` and ``w%dqdt_3d`` in place.  ``DeviceDomain`` is
that subset, held as CUDA tensors (device pointers cross the C ABI) or numpy
arrays (host pointers; the library stages them).  Arrays keep the Fortran
layout (i fastest, then k, then j), i.e. numpy/torch shape (ny, nz, nx).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import _capi

METRIC_FIELDS = _capi.METRIC_FIELDS


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def ptr(a) -> int:
    """Raw address of a contiguous torch tensor or numpy array."""
    if a is None:
        return 0
    if _is_torch(a):
        assert a.is_contiguous(), "arrays crossing the C ABI must be contiguous"
        return a.data_ptr()
    assert a.flags.c_contiguous, "arrays crossing the C ABI must be contiguous"
    return a.ctypes.data


def mem_kind(a) -> int:
    if _is_torch(a):
        return _capi.MEM_DEVICE if a.is_cuda else _capi.MEM_HOST
    return _capi.MEM_HOST


@dataclasses.dataclass
class DeviceDomain:
    nx: int
    ny: int
    nz: int
    dx: float
    nest_indx: int
    metrics: dict                 # METRIC_FIELDS -> array
    density: object               # (ny, nz, nx)
    u_dqdt: object                # (ny, nz, nx+1)
    v_dqdt: object                # (ny+1, nz, nx)
    w_dqdt: object                # (ny, nz, nx)
    wind_alpha: object            # (ny, nz, nx)
    u: object = None              # data_3d winds, read by calc_divergence(use_dqdt=False)
    v: object = None
    w: object = None

    @property
    def ncell(self) -> int:
        return self.nx * self.ny * self.nz

    @staticmethod
    def from_case(case, device: str = "cuda", nest_indx: int = 1) -> "DeviceDomain":
        d = case.domain
        if device == "cpu":
            conv = lambda a: np.ascontiguousarray(a, dtype=np.float32).copy()  # noqa: E731
        else:
            import torch
            conv = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)  # noqa: E731
        metrics = {n: conv(getattr(d, n)) for n in METRIC_FIELDS}
        return DeviceDomain(nx=d.nx, ny=d.ny, nz=d.nz, dx=float(d.dx), nest_indx=nest_indx, metrics=metrics,
                            density=conv(d.density), u_dqdt=conv(case.u), v_dqdt=conv(case.v), w_dqdt=conv(case.w),
                            wind_alpha=conv(case.alpha))

    def set_winds(self, u, v, w) -> None:
        """Overwrite the dqdt winds in place (keeps the device buffers)."""
        for dst, src in ((self.u_dqdt, u), (self.v_dqdt, v), (self.w_dqdt, w)):
            if _is_torch(dst):
                import torch
                dst.copy_(src if _is_torch(src) else torch.from_numpy(np.ascontiguousarray(src, np.float32)))
            else:
                dst[...] = src
