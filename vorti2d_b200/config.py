"""Case configuration (drop-in for ``vorti2d.Config``, vorti2d/config.py:12-169).

Every field of the reference keeps its name, default and meaning.  The GPU
solver adds a few defaulted knobs at the end (precision, preconditioner,
Krylov limits); a reference Config script runs unchanged.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, asdict


@dataclass
class Config:
    # ---------------------------------------------------------------- physics
    re: float = 60.0
    # ------------------------------------------------------- time integration
    steady: bool = False
    dt_phys: float = 0.2
    t_start: float = 0.0
    t_end: float = 50.0
    dtau: float = math.inf
    # ------------------------------------------- inner (pseudo-time) controls
    pseudo_tol: float = 1.0e-10
    max_pseudo_iter: int = 200
    # ------------------------------------------------------ rotation schedule
    rot_speed: float = 0.0
    rot_until: float = 0.0
    # --------------------------------------------------------- far-field BC
    farfield_bc: str = "dirichlet"
    # -------------------------------------------------------- angle of attack
    alpha_deg: float = 0.0
    # ------------------------------------------------------- parallel solver
    distributed: bool = False
    # -------------------------------------------------------- linear solver
    linsolve: str = "mumps"
    ksp_rtol: float = 1.0e-10
    ksp_restart: int = 200
    ilu_fill: int = 1
    asm_overlap: int = 1
    # ------------------------------------------------------------------ mesh
    mesh_xg: str = "xg.csv"
    mesh_yg: str = "yg.csv"
    mesh_cgns: str | None = None
    inner_rad: float = 0.5
    outer_rad: float = 50.0
    # ---------------------------------------------------------------- output
    out_dir: str = "out"
    save_fields_every: int = 1
    verbose: bool = True
    write_csv: bool = True
    write_xdmf: bool = True
    # ---------------------------------------------------- force coefficients
    compute_forces: bool = True
    ref_length: float | None = None
    moment_center: tuple[float, float] = (0.0, 0.0)
    # --------------------------------------------------------------- restart
    restart_in: str | None = None
    restart_out: str = "restart.npz"
    restart_every: int = 0
    # ------------------------------------------------------------- GPU knobs
    precision: str = "fp64"
    """``"fp64"``: FP64 GMRES.  ``"mixed"``: FP32 SpMV / preconditioner /
    Krylov vectors inside an FP64 defect correction (FP64 residual, metrics,
    Jacobian entries, Gram-Schmidt sums and forces)."""
    precond: str = "lu"
    """Krylov preconditioner: ``"lu"`` (multifrontal LU of each Newton
    Jacobian on the device, FP32 factors in the mixed form; converges in a few
    iterations like the reference's direct MUMPS solve), ``"bjacobi"`` (2x2
    psi/ome node blocks; cheap per iteration, but pure Newton systems
    (dtau = inf) converge slowly or not at all) or ``"none"``."""
    krylov_max_it: int = 5000
    inner_rtol: float = 1.0e-5
    """Mixed precision: relative residual reduction asked of each FP32 cycle."""
    lu_reuse_its: int = 0
    """LU preconditioner: 0 factors every Newton Jacobian; k > 0 keeps the
    factors across the Newton iterations of one time step while the last
    solve with them needed at most k Krylov iterations (each Newton step is
    still solved to ``ksp_rtol``)."""
    lu_reuse_steps: bool = False
    """LU preconditioner with ``lu_reuse_its > 0``: keep the factors across
    time steps and ``set_state`` too (the same iteration rule decides when to
    refactor)."""
    lu_factors: str = "fp32"
    """LU preconditioner in the mixed form: ``"fp32"`` factors in FP32;
    ``"fp64"`` factors in FP64 and rounds the factors to FP32 for the FP32
    solve (more accurate pivots and updates, the same bytes per solve).  The
    FP64 form always factors in FP64."""
    lu_item_rows: list | None = None
    """LU preconditioner solve: rows per work item on each tree level (0:
    whole fronts; R > 0: R rows; R < 0: -R rows after one gather item per
    front), e.g. from ``vorti2d_b200.tune``; None keeps the default split."""
    lu_solve: str = "flow"
    """LU preconditioner solve: ``"flow"`` runs each application as one
    dataflow launch over the whole front tree; ``"levels"`` as one launch per
    tree level and sweep (same arithmetic, same results)."""
    raise_on_linear_failure: bool = True
    """Raise if a Krylov solve misses ``ksp_rtol`` (the reference raises on a
    failed PETSc solve, vorti2d/petsc_solver.py:103-105)."""

    # reference helpers (vorti2d/config.py:139-166)
    def inv_dtau(self) -> float:
        return 0.0 if math.isinf(self.dtau) else 1.0 / self.dtau

    def inv_2dt(self) -> float:
        return 0.0 if self.steady else 1.0 / (2.0 * self.dt_phys)

    def cos_alpha(self) -> float:
        return math.cos(math.radians(self.alpha_deg))

    def sin_alpha(self) -> float:
        return math.sin(math.radians(self.alpha_deg))

    def ff_bc_code(self) -> int:
        codes = {"dirichlet": 0, "outflow": 1, "outflow_psi": 2}
        try:
            return codes[self.farfield_bc.lower()]
        except KeyError:
            raise ValueError(
                f"unknown farfield_bc={self.farfield_bc!r}; "
                f"choose one of {sorted(codes)}")

    def u_rot(self, t: float) -> float:
        if self.steady:
            return self.rot_speed
        return self.rot_speed if t <= self.rot_until else 0.0

    def to_dict(self) -> dict:
        return asdict(self)

    # GPU helpers
    def precision_code(self) -> int:
        codes = {"fp64": 0, "mixed": 1}
        try:
            return codes[self.precision.lower()]
        except KeyError:
            raise ValueError(f"unknown precision={self.precision!r}; choose one of {sorted(codes)}")

    def precond_code(self) -> int:
        codes = {"none": 0, "bjacobi": 1, "lu": 2}
        try:
            return codes[self.precond.lower()]
        except KeyError:
            raise ValueError(f"unknown precond={self.precond!r}; choose one of {sorted(codes)}")

    def check_linsolve(self):
        """The reference's linsolve names all select the device GMRES here
        (MUMPS / PETSc are not part of the GPU path)."""
        known = {"mumps", "gmres_asm", "gmres_jacobi", "gpu", "gmres_fs", "fieldsplit",
                 "gmres_amgx", "gpu_amgx"}
        if self.linsolve.lower() not in known:
            raise ValueError(
                f"unknown linsolve={self.linsolve!r} (choose 'mumps', 'gmres_asm',"
                f" 'gmres_jacobi'/'gpu', 'gmres_amgx', or 'gmres_fs')")
