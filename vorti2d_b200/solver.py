"""The vorti2d driver on the GPU (drop-in for ``vorti2d.Solver`` / ``run``,
vorti2d/solver.py:32-296).

Outer loop: physical time (BDF2; one pass when steady).  Inner loop: Newton
iterations until ||dq||_2/(2N) <= pseudo_tol or max_pseudo_iter.  Every
Newton iteration runs on the device (libvorti2d_b200: assembly into a fixed
CSR, GMRES(m), q += dq); the state stays in HBM and is copied to the host
only for output, restart files and attribute access.
"""
from __future__ import annotations

import ctypes
import math
import os
import time

import numpy as np

from . import _lib
from . import fields_io
from . import forces as forcesmod
from . import mesh as meshmod
from . import restart as restartmod
from ._lib import check, dptr, lib
from .config import Config

_PROFILE = bool(os.environ.get("VORTI2D_TIMING"))


def solver_params(cfg: Config) -> _lib.SolverParams:
    p = _lib.SolverParams()
    p.re = float(cfg.re)
    p.invdtau = cfg.inv_dtau()
    p.inv2dt = cfg.inv_2dt()
    p.ca = cfg.cos_alpha()
    p.sa = cfg.sin_alpha()
    p.ff_bc = cfg.ff_bc_code()
    k = _lib.krylov_defaults()
    k.restart = int(cfg.ksp_restart)
    k.rtol = float(cfg.ksp_rtol)
    k.max_it = int(cfg.krylov_max_it)
    k.precision = cfg.precision_code()
    k.precond = cfg.precond_code()
    k.inner_rtol = float(cfg.inner_rtol)
    k.lu_reuse_its = int(cfg.lu_reuse_its)
    k.lu_reuse_steps = int(bool(cfg.lu_reuse_steps))
    k.lu_solve = {"flow": 0, "levels": 1}[cfg.lu_solve]
    k.lu_factor64 = {"fp32": 0, "fp64": 1}[cfg.lu_factors]
    p.krylov = k
    return p


class DeviceState:
    """Owns one device handle (mesh, metrics, state, CSR, Krylov workspace)."""

    def __init__(self, xg, yg, cfg: Config):
        xg = np.asfortranarray(xg, dtype=np.float64)
        yg = np.asfortranarray(yg, dtype=np.float64)
        self.imax, self.jmax = xg.shape
        self.N = self.imax * self.jmax
        self.params = solver_params(cfg)
        h = ctypes.c_void_p()
        check(lib().v2d_solver_create(self.imax, self.jmax, dptr(xg), dptr(yg),
                                      ctypes.byref(self.params), ctypes.byref(h)), "Solver")
        self.h = h

    def metrics(self):
        outs = [np.zeros(self.N) for _ in range(10)]
        arr = (ctypes.POINTER(ctypes.c_double) * 10)(*[dptr(o) for o in outs])
        check(lib().v2d_solver_get_metrics(self.h, arr), "get_metrics")
        return outs

    def get_state(self, out=None):
        """psi, ome, omeold, omeoldold as flat float64 arrays.  ``out``: four
        caller-owned C-contiguous float64 arrays of imax*jmax entries (e.g.
        views of pinned host buffers) to copy into instead of new arrays."""
        if out is None:
            outs = [np.zeros(self.N) for _ in range(4)]
        else:
            outs = list(out)
            if len(outs) != 4:
                raise ValueError("get_state: out needs four arrays (psi, ome, omeold, omeoldold)")
            for o in outs:
                if (not isinstance(o, np.ndarray) or o.dtype != np.float64 or o.size != self.N
                        or not o.flags.c_contiguous or not o.flags.writeable):
                    raise ValueError(f"get_state: each out array must be a writable C-contiguous "
                                     f"float64 array of imax*jmax = {self.N} entries")
        check(lib().v2d_solver_get_state(self.h, *[dptr(o) for o in outs]), "get_state")
        return outs

    def set_re(self, re: float):
        """Change the Reynolds number of the handle's Newton system (the
        state, pattern and workspaces stay; old LU factors are not reused)."""
        if not (np.isfinite(re) and re > 0):
            raise ValueError(f"set_re: Re must be finite and positive, got {re}")
        self.params.re = float(re)
        check(lib().v2d_solver_set_params(self.h, ctypes.byref(self.params)), "set_params")

    def set_invdtau(self, invdtau: float):
        """Change the pseudo-time term 1/dtau that the Newton Jacobian's
        diagonal carries (0: plain Newton)."""
        if not (np.isfinite(invdtau) and invdtau >= 0):
            raise ValueError(f"set_invdtau: 1/dtau must be finite and >= 0, got {invdtau}")
        self.params.invdtau = float(invdtau)
        check(lib().v2d_solver_set_params(self.h, ctypes.byref(self.params)), "set_params")

    def set_state(self, psi, ome, omeold, omeoldold):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (psi, ome, omeold, omeoldold)]
        for a in arrs:
            if a.size != self.N:
                raise ValueError(f"state arrays must have imax*jmax = {self.N} entries")
        check(lib().v2d_solver_set_state(self.h, *[dptr(a) for a in arrs]), "set_state")

    def newton(self, urot: float):
        res = ctypes.c_double()
        st = _lib.LinStats()
        code = lib().v2d_solver_newton(self.h, float(urot), ctypes.byref(res), ctypes.byref(st))
        return code, res.value, st

    def shift_history(self):
        check(lib().v2d_solver_shift_history(self.h), "shift_history")

    def velocity(self, want_mag=False):
        N = self.N
        u, v = np.empty(N), np.empty(N)
        mag = np.empty(N) if want_mag else None
        check(lib().v2d_solver_velocity(self.h, dptr(u), dptr(v), dptr(mag) if want_mag else None),
              "velocity")
        return (u, v, mag) if want_mag else (u, v)

    def forces(self, re, ref_length, moment_ref):
        out = np.zeros(10)
        rl = -1.0 if ref_length is None else float(ref_length)
        check(lib().v2d_solver_forces(self.h, float(re), rl, float(moment_ref[0]),
                                      float(moment_ref[1]), dptr(out)), "forces")
        return forcesmod.ForceCoeffs.from_array(out)

    def system(self, urot=None):
        """(indptr, indices, data, b) of the current Newton system; assembles
        first when urot is given."""
        if urot is not None:
            check(lib().v2d_solver_assemble(self.h, float(urot)), "assemble")
        nnz = ctypes.c_longlong()
        check(lib().v2d_solver_nnz(self.h, ctypes.byref(nnz)))
        n = 2 * self.N
        ip = np.zeros(n + 1, dtype=np.intc)
        ix = np.zeros(nnz.value, dtype=np.intc)
        dv = np.zeros(nnz.value)
        b = np.zeros(n)
        check(lib().v2d_solver_export_system(self.h, _lib.iptr(ip), _lib.iptr(ix), dptr(dv),
                                             dptr(b)), "export_system")
        return ip, ix, dv, b

    def close(self):
        if getattr(self, "h", None):
            lib().v2d_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Replicated-state solver (vorti2d/solver.py:32-283) with the state in HBM.

    ``mesh=(xg, yg)`` may be passed to skip reading ``cfg.mesh_xg/mesh_yg``.
    """

    def __init__(self, config: Config, mesh=None):
        self.cfg = config
        self.rank, self.size = 0, 1
        self.restarted = False
        self._t_kernel = 0.0
        self._mesh = mesh
        self.newton_log = []     # (t, newton its, krylov its, res)
        self._setup()

    def _log(self, msg: str):
        if self.rank == 0 and self.cfg.verbose:
            print(msg, flush=True)

    def _setup(self):
        cfg = self.cfg
        cfg.check_linsolve()
        if self._mesh is not None:
            xg, yg = (np.asarray(a, dtype=np.float64) for a in self._mesh)
        elif cfg.mesh_cgns:
            xg, yg = meshmod.load_cgns_ogrid(cfg.mesh_cgns, verbose=cfg.verbose)
        else:
            xg, yg = meshmod.load_mesh(cfg.mesh_xg, cfg.mesh_yg)
        self.xg, self.yg = xg, yg
        self.imax, self.jmax = xg.shape
        self.ndof = self.imax * self.jmax
        self.dksi = 1.0 / (self.imax - 1)
        self.deta = 1.0 / (self.jmax - 1)
        self._ff_bc = cfg.ff_bc_code()
        self._ca = cfg.cos_alpha()
        self._sa = cfg.sin_alpha()
        self.dev = DeviceState(xg, yg, cfg)
        if cfg.lu_item_rows is not None and cfg.precond.lower() == "lu":
            from .tune import set_item_rows
            set_item_rows(self, cfg.lu_item_rows)
        (self.jac, self.alfa, self.beta, self.gama, self.pmet, self.qmet, self.detadx,
         self.detady, self.xphys, self.yphys) = self.dev.metrics()
        self.r0, self.r1 = 0, 2 * self.ndof
        self.maxnnz = (self.r1 - self.r0) * 13
        self._host_state = None
        self._init_state()
        self._log(f"vorti2d_b200: mesh {self.imax}x{self.jmax}  ndof={self.ndof}  "
                  f"mode={'steady' if cfg.steady else 'unsteady'}  "
                  f"precision={cfg.precision}")

    def _init_state(self):
        cfg = self.cfg
        if cfg.restart_in:
            st = restartmod.load_restart(cfg.restart_in, self.imax, self.jmax)
            self.dev.set_state(st.psi, st.ome, st.omeold, st.omeoldold)
            self.t, self.step = float(st.t), int(st.step)
            self.restarted = True
            self._log(f"  restarted from {cfg.restart_in}: t={self.t}, step={self.step}")
        else:
            # the device handle starts from zeros with the far-field
            # streamfunction (vorti2d/solver.py:103-112)
            self.t = cfg.t_start
            self.step = 0
        self._host_state = None

    # ---------------------------------------------------------- state access
    def _state(self):
        if self._host_state is None:
            self._host_state = self.dev.get_state()
        return self._host_state

    @property
    def psi(self):
        return self._state()[0]

    @property
    def ome(self):
        return self._state()[1]

    @property
    def omeold(self):
        return self._state()[2]

    @property
    def omeoldold(self):
        return self._state()[3]

    def get_state(self, out=None):
        """Copy the device state (psi, ome, omeold, omeoldold; flat, i fastest)
        to the host; ``out`` names four caller-owned float64 arrays to fill."""
        if out is None:
            return [a.copy() for a in self._state()]
        return self.dev.get_state(out)

    def set_state(self, psi, ome, omeold, omeoldold):
        self.dev.set_state(psi, ome, omeold, omeoldold)
        self._host_state = None

    # --------------------------------------------------------------- solving
    def _assemble_and_solve_once(self, invdtau, inv2dt, urot):
        """vorti2d/solver.py:117-134 on the device; returns ||dq||/(2N)."""
        t0 = time.perf_counter() if _PROFILE else 0.0
        code, res, st = self.dev.newton(urot)
        self._host_state = None
        if _PROFILE:
            self._t_kernel += time.perf_counter() - t0
        self._last_lin = st
        if code == _lib.V2D_ENOTCONVERGED and not self.cfg.raise_on_linear_failure:
            return res
        check(code, "Newton iteration")
        return res

    def _pseudo_solve(self, t, invdtau, inv2dt, urot):
        """vorti2d/solver.py:136-145."""
        cfg = self.cfg
        res, it, kits = 1.0e5, 0, 0
        res_log = []
        while res > cfg.pseudo_tol and it < cfg.max_pseudo_iter:
            res = self._assemble_and_solve_once(invdtau, inv2dt, urot)
            it += 1
            kits += self._last_lin.iterations
            res_log.append(math.log10(res) if res > 0 else -300.0)
        self.newton_log.append((t, it, kits, res))
        return res, it, res_log

    def advance(self, t):
        """One physical step at time t (vorti2d/solver.py:182-191)."""
        cfg = self.cfg
        res, it, res_log = self._pseudo_solve(t, cfg.inv_dtau(), cfg.inv_2dt(), cfg.u_rot(t))
        if not cfg.steady:
            self.dev.shift_history()
            self._host_state = None
        self.t = t
        self.step += 1
        return res, it, res_log

    def times(self):
        cfg = self.cfg
        if cfg.steady:
            return [cfg.t_start]
        start = self.t + cfg.dt_phys if self.restarted else cfg.t_start
        nsteps = int(round((cfg.t_end - start) / cfg.dt_phys)) + 1
        return [start + m * cfg.dt_phys for m in range(max(nsteps, 0))]

    # ------------------------------------------------------------------- run
    def run(self):
        """vorti2d/solver.py:148-224 (XDMF/HDF5 output needs h5py, which
        vorti2d_b200 does not depend on: ``write_xdmf`` is ignored with a
        notice)."""
        cfg = self.cfg
        if cfg.write_xdmf and cfg.verbose:
            self._log("  note: write_xdmf ignored (XDMF/HDF5 output is not part of vorti2d_b200)")
        # the output folder and the grid are written on every run, as the
        # reference does (vorti2d/solver.py:150-160)
        fields_io.ensure_dirs(cfg.out_dir)
        fields_io.write_grid(cfg.out_dir, self.xg, self.yg)
        forces_path = os.path.join(cfg.out_dir, "forces.csv")
        if cfg.compute_forces and (not self.restarted or not os.path.exists(forces_path)):
            fields_io.init_force_history(cfg.out_dir, forcesmod.FORCE_COLUMNS)
        t_wall0 = time.time()
        local_step = 0
        for t in self.times():
            res, it, res_log = self.advance(t)
            local_step += 1
            time_idx = 0 if cfg.steady else int(round(t / cfg.dt_phys))
            self._log(f"  t={t:8.3f}  inner_iters={it:3d}  res={res:.3e}  step={self.step}")
            save_now = cfg.steady or local_step % cfg.save_fields_every == 0
            if cfg.compute_forces:
                fc = self.force_coeffs()
                row = {"t": t, **fc.to_dict()}
                fields_io.append_force_history(cfg.out_dir, forcesmod.FORCE_COLUMNS, row)
                self._log(f"           Cd={fc.cd:+.5f}  Cl={fc.cl:+.5f}  Cm={fc.cm:+.5f}")
            if save_now and cfg.write_csv:
                fields_io.write_fields(cfg.out_dir, time_idx, self.psi, self.ome)
                fields_io.write_residual_history(cfg.out_dir, time_idx, res_log)
            if cfg.restart_every and not cfg.steady and local_step % cfg.restart_every == 0:
                self._write_restart()
        self._write_restart()
        self._log(f"vorti2d_b200: done in {time.time() - t_wall0:.2f}s, final t={self.t}")
        return self

    def _write_restart(self):
        path = self.cfg.restart_out
        if not os.path.isabs(path):
            os.makedirs(self.cfg.out_dir, exist_ok=True)
            path = os.path.join(self.cfg.out_dir, path)
        st = restartmod.RestartState(self.psi, self.ome, self.omeold, self.omeoldold, self.t,
                                     self.step, self.imax, self.jmax, self.cfg.re)
        restartmod.save_restart(path, st)

    # ----------------------------------------------------------- accessors
    def field_2d(self, name: str) -> np.ndarray:
        arr = {"psi": self.psi, "ome": self.ome}[name]
        return arr.reshape(self.jmax, self.imax).T

    def force_coeffs(self) -> forcesmod.ForceCoeffs:
        """Cl/Cd/Cm of the current state, integrated on the device
        (vorti2d/solver.py:272-283 -> vorti2d/forces.py:82-194)."""
        cfg = self.cfg
        return self.dev.forces(cfg.re, cfg.ref_length, cfg.moment_center)

    def velocity(self, want_mag: bool = False):
        """Cartesian velocity of the current state, on the device
        (vorti2d/velocity.py:76-93)."""
        return self.dev.velocity(want_mag)

    def close(self):
        self.dev.close()


def run(config: Config, mesh=None):
    """vorti2d/solver.py:286-296.  ``distributed=True`` (the reference's DMDA
    multi-rank solver) has no separate path here: one GPU holds the whole
    replicated state, so it runs the same device solver."""
    return Solver(config, mesh=mesh).run()
