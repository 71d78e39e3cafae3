"""sw2d_b200: SW2D's single-porosity explicit finite-volume step on the NVIDIA B200.

Modules:
  case       -- SW2D case folders (geometry.sw2d v2, maps, boundary series, input.solv)
  mesh       -- synthetic triangle meshes with the reference's geometry conventions
  workloads  -- seeded synthetic cases (dam break, Gaussian bumps, feature channel)
  capi       -- ctypes view of include/sw2d_b200.h and the CUDA library loader
  solver     -- SpModel, the host-side mirror of the reference's swSp interface
  tuning     -- launch-configuration autotuner with a JSON cache
  assimilation -- friction assimilation over the GPU adjoint (the reference's swSpE_minimize)
  porosity   -- porosity assimilation with the reference's differentiated step (swSpE, its
                input.solv keys, observation files, PorosityProblem and run_minimization)
  batch      -- ensembles of independent simulations advanced together (one graph launch)
  autograd   -- torch.autograd bridge to the replayed cost and its adjoint (imported on demand)
"""
from . import build, case, mesh, workloads, capi, solver, tuning, assimilation, batch, porosity, closure, porosity_mapper  # noqa: F401
from .case import Case, read_case, write_case  # noqa: F401
from .solver import SpModel, Sw2dError  # noqa: F401
from .batch import Batch  # noqa: F401

__all__ = ["case", "mesh", "workloads", "capi", "solver", "assimilation", "batch", "porosity", "Case", "read_case",
           "write_case", "SpModel", "Sw2dError", "Batch"]
