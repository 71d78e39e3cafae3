"""sw2d_b200: SW2D's single-porosity explicit finite-volume step on the NVIDIA B200.

Modules:
  case       -- SW2D case folders (geometry.sw2d v2, maps, boundary series, input.solv)
  mesh       -- synthetic triangle meshes with the reference's geometry conventions
  workloads  -- seeded synthetic cases (dam break, Gaussian bumps, feature channel)
  capi       -- ctypes view of include/sw2d_b200.h and the CUDA library loader
  solver     -- SpModel, the host-side mirror of the reference's swSp interface
  tuning     -- launch-configuration autotuner with a JSON cache
"""
from . import build, case, mesh, workloads, capi, solver, tuning  # noqa: F401
from .case import Case, read_case, write_case  # noqa: F401
from .solver import SpModel, Sw2dError  # noqa: F401

__all__ = ["case", "mesh", "workloads", "capi", "solver", "Case", "read_case", "write_case", "SpModel", "Sw2dError"]
