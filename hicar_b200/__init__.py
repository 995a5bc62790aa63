"""hicar_b200 -- B200 (sm_100a) implementation of HICAR's iterative
mass-conserving wind solver (module wind_iterative), behind a C ABI
(include/hicarw.h) that HICAR's Fortran calls through ISO_C_BINDING.

Python modules mirror the reference's interface for this path:
  wind_iterative  init_iter_winds / calc_iter_winds / finalize_iter_winds / probe_*
  wind            calc_divergence / calibrate_projection_operator / update_winds_iterative
  domain          the domain fields the solver reads and writes
  cases           seeded synthetic domains (terrain, Gal-Chen metrics, winds)
"""
from . import _capi, cases  # noqa: F401

__all__ = ["_capi", "cases", "wind_iterative", "wind", "domain", "build"]
