"""vorti2d_b200: B200-native implementation of vorti2d's implicit
Newton / dual-time hot path (metrics, coupled psi-omega assembly into CSR,
GMRES(m) with block Jacobi), behind the reference's ``core`` / ``Config`` /
``run`` / ``MumpsSolver`` interfaces.  Kernels: libvorti2d_b200.so (sm_100a).
"""
from __future__ import annotations

from .core import vorti2d_core as core
from . import mesh
from .config import Config
from .mesh import (generate_cylinder, generate_naca0012, load_cgns_ogrid, load_mesh,
                   save_mesh)
from .solver import Solver, run
from .forces import compute_force_coeffs, ForceCoeffs
from . import velocity
from .velocity import compute_velocity
from .petsc_solver import GpuLinearSolver, MumpsSolver

__all__ = [
    "Config", "Solver", "run", "generate_cylinder", "generate_naca0012", "load_mesh",
    "load_cgns_ogrid", "save_mesh", "compute_force_coeffs", "ForceCoeffs", "mesh", "core",
    "GpuLinearSolver", "MumpsSolver", "velocity", "compute_velocity",
]

__version__ = "0.1.0"
