"""Linear-solver seam: drop-in for ``vorti2d.petsc_solver.MumpsSolver``
(vorti2d/petsc_solver.py:37-132), solved on the GPU.

Same five methods: ``row_range``, ``assemble``, ``solve``, ``timings``,
``destroy``.  One process owns the whole system (r0 = 0, r1 = n); the first
``assemble`` fixes the canonical CSR pattern on the device, later calls only
refresh values (as the reference's preallocated pattern does).

The default preconditioner is "lu": every solve factors the assembled matrix
with the device multifrontal LU and refines with GMRES to ``rtol``, which is
what the reference's MUMPS direct solve (petsc_solver.py:55-61) delivers.  The
LU's ordering needs the O-grid shape: pass ``grid=(imax, jmax)``, or let the
first ``assemble`` recognise it from the pattern.  "bjacobi" and "none" need
no grid but converge slowly or not at all on pure-Newton systems.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr, lib

_PROFILE = bool(os.environ.get("VORTI2D_TIMING"))


class GpuLinearSolver:
    """``MumpsSolver(n, comm)`` interface on the device.

    block_layout: 1 pairs rows (q, q + n/2) into 2x2 blocks (the replicated
    field-blocked system), 2 pairs (2q, 2q+1) (node-interleaved / DMDA
    ordering), 0 point Jacobi.
    """

    def __init__(self, n: int, comm=None, block_layout: int = 1, restart: int = 30,
                 rtol: float = 1e-10, max_it: int = 5000, precision: str = "fp64",
                 precond: str = "lu", inner_rtol: float = 1e-5, grid=None,
                 lu_reuse_its: int = 0):
        self.comm = comm
        self.n = int(n)
        self.r0, self.r1 = 0, self.n
        self.nloc = self.n
        p = _lib.krylov_defaults()
        p.restart = int(restart)
        p.rtol = float(rtol)
        p.max_it = int(max_it)
        p.precision = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        p.precond = {"none": _lib.PC_NONE, "bjacobi": _lib.PC_BJACOBI, "lu": _lib.PC_LU}[precond]
        p.inner_rtol = float(inner_rtol)
        p.lu_reuse_its = int(lu_reuse_its)
        self._params = p
        h = ctypes.c_void_p()
        check(lib().v2d_linsys_create(self.n, int(block_layout), ctypes.byref(p), ctypes.byref(h)),
              "MumpsSolver")
        self._h = h
        if grid is not None:
            check(lib().v2d_linsys_set_grid(h, int(grid[0]), int(grid[1])), "MumpsSolver(grid)")
        self.t_csr = self.t_solve = self.t_gather = 0.0
        self.n_solves = 0
        self.last_stats = None

    def row_range(self):
        """Owned global row range [r0, r1) (vorti2d/petsc_solver.py:72-74)."""
        return self.r0, self.r1

    def assemble(self, coo_i, coo_j, coo_v, bvec):
        """vorti2d/petsc_solver.py:76-95."""
        t0 = time.perf_counter() if _PROFILE else 0.0
        ci = np.ascontiguousarray(coo_i, dtype=np.intc)
        cj = np.ascontiguousarray(coo_j, dtype=np.intc)
        cv = np.ascontiguousarray(coo_v, dtype=np.float64)
        b = np.ascontiguousarray(bvec, dtype=np.float64)
        if not (ci.size == cj.size == cv.size):
            raise ValueError("coo_i, coo_j, coo_v must have the same length")
        if b.size != self.n:
            raise ValueError(f"bvec must have {self.n} entries (got {b.size})")
        check(lib().v2d_linsys_assemble(self._h, iptr(ci), iptr(cj), dptr(cv), ci.size, dptr(b)),
              "MumpsSolver.assemble")
        if _PROFILE:
            self.t_csr += time.perf_counter() - t0

    def solve(self) -> np.ndarray:
        """Solve A x = b; return the full solution (vorti2d/petsc_solver.py:97-115).
        Raises RuntimeError if GMRES misses the tolerance (the reference raises
        on a failed PETSc solve)."""
        t0 = time.perf_counter() if _PROFILE else 0.0
        x = np.zeros(self.n)
        st = _lib.LinStats()
        code = lib().v2d_linsys_solve(self._h, dptr(x), ctypes.byref(st))
        self.last_stats = st
        check(code, "MumpsSolver.solve")
        if _PROFILE:
            self.t_solve += time.perf_counter() - t0
        self.n_solves += 1
        return x

    def csr(self):
        """Canonical CSR (indptr, indices, data) of the assembled matrix."""
        nnz = ctypes.c_longlong()
        check(lib().v2d_linsys_nnz(self._h, ctypes.byref(nnz)))
        ip = np.zeros(self.n + 1, dtype=np.intc)
        ix = np.zeros(nnz.value, dtype=np.intc)
        dv = np.zeros(nnz.value)
        check(lib().v2d_linsys_csr(self._h, iptr(ip), iptr(ix), dptr(dv)))
        return ip, ix, dv

    def timings(self) -> dict:
        """vorti2d/petsc_solver.py:117-125 (one process: no max over ranks)."""
        return {"csr_assemble": self.t_csr, "linsolve": self.t_solve,
                "gather_toall": self.t_gather, "n_solves": self.n_solves}

    def destroy(self):
        if getattr(self, "_h", None):
            lib().v2d_linsys_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


MumpsSolver = GpuLinearSolver
