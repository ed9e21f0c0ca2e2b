"""Batched steady sweeps: many independent steady solves of uneven grid sizes
(cylinders and NACA-0012 sections over a range of Reynolds numbers and
angles of attack) on one GPU.

``run_sweep_batched`` (the default) advances all instances by Newton
together: their systems are the diagonal blocks of one block-diagonal system,
so each Newton iteration is one assembly launch over all instances, one
multifrontal factorization over the forest of their separator trees, GMRES
on the combined system and one update launch (``v2d_batch_*``).  Converged
and diverging instances are frozen and stop contributing work.

``run_sweep`` is the earlier form: every instance its own device handle and
CUDA stream, driven by a pool of host threads.

Plain Newton from the free stream (the reference's steady method) does not
reach a steady state at the higher Reynolds numbers of a sweep: each instance
reports whether it converged, and the sweep's throughput is counted both in
Newton iterations (the work done) and in converged solves.
"""
from __future__ import annotations

import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .config import Config
from .mesh import generate_cylinder, generate_naca0012


@dataclass
class Case:
    name: str
    xg: np.ndarray
    yg: np.ndarray
    re: float
    alpha_deg: float
    ref_length: float | None = None


@dataclass
class CaseResult:
    name: str
    re: float
    alpha_deg: float
    nodes: int
    converged: bool
    newton_iters: int
    res: float
    krylov_iters: int = 0
    diverged: bool = False
    re_reached: float = math.nan   # last Reynolds number solved (continuation)
    rungs: int = 0                 # Reynolds numbers attempted (1 without continuation)
    cd: float = math.nan
    cl: float = math.nan
    cm: float = math.nan
    seconds: float = 0.0
    error: str = ""


def sweep_cases(seed: int = 0, n_each: int = 32):
    """The batched sweep: n_each cylinders at 129x129, n_each at 181x181 and
    n_each NACA-0012 sections at 257x129 (open trailing edge, far field 30
    chords); Re ~ U[50, 1000], alpha ~ U[-8, 8] degrees from one seeded
    generator."""
    rng = np.random.default_rng(seed)
    meshes = {"cyl129": generate_cylinder(129, 129), "cyl181": generate_cylinder(181, 181),
              "naca257x129": generate_naca0012(257, 129)}
    cases = []
    for kind in ("cyl129", "cyl181", "naca257x129"):
        xg, yg = meshes[kind]
        for k in range(n_each):
            re = float(rng.uniform(50.0, 1000.0))
            alpha = float(rng.uniform(-8.0, 8.0))
            cases.append(Case(f"{kind}_{k:02d}", xg, yg, re, alpha,
                              1.0 if kind.startswith("naca") else None))
    return cases


def _config(case: Case, precision: str, max_newton: int, pseudo_tol: float,
            krylov_max_it: int, **kw) -> Config:
    return Config(re=case.re, alpha_deg=case.alpha_deg, steady=True, verbose=False,
                  write_csv=False, write_xdmf=False, compute_forces=False,
                  pseudo_tol=pseudo_tol, max_pseudo_iter=max_newton, ksp_rtol=1e-10,
                  krylov_max_it=krylov_max_it, precision=precision,
                  ref_length=case.ref_length, raise_on_linear_failure=False, **kw)


@dataclass
class SweepResult:
    results: list = field(default_factory=list)
    setup_s: float = 0.0
    solve_s: float = 0.0
    workers: int = 0
    shared_krylov: int | None = None   # batched: GMRES iterations of the combined system

    @property
    def converged(self) -> int:
        return sum(r.converged for r in self.results)

    @property
    def newton_iters(self) -> int:
        return sum(r.newton_iters for r in self.results)

    @property
    def krylov_iters(self) -> int:
        if self.shared_krylov is not None:
            return self.shared_krylov
        return sum(r.krylov_iters for r in self.results)

    @property
    def solves_per_s(self) -> float:
        return self.converged / self.solve_s if self.solve_s > 0 else 0.0

    @property
    def newton_per_s(self) -> float:
        return self.newton_iters / self.solve_s if self.solve_s > 0 else 0.0


def re_ladder(re_target: float, re_start: float, factor: float | None) -> list:
    """Reynolds numbers of a natural-parameter continuation: re_start,
    re_start*factor, ... while below re_target, then re_target itself.  No
    continuation (``factor`` None or 0, or re_target <= re_start): the
    target alone."""
    if not (math.isfinite(re_target) and re_target > 0):
        raise ValueError(f"re_ladder: target Re must be finite and positive, got {re_target}")
    if not factor or re_target <= re_start:
        return [float(re_target)]
    if not (factor > 1.0 and math.isfinite(factor)):
        raise ValueError(f"re_ladder: factor must be > 1, got {factor}")
    if not re_start > 0:
        raise ValueError(f"re_ladder: start Re must be positive, got {re_start}")
    out, re = [], float(re_start)
    while re < re_target:
        out.append(re)
        re *= factor
    out.append(float(re_target))
    return out


def solve_case(s, r: CaseResult, ladder, max_newton: int, pseudo_tol: float,
               rung_tol: float, diverge_factor: float) -> float:
    """Steady Newton solves of one instance along ``ladder`` (its Reynolds
    numbers, last = the case's own).  ``s`` is a Solver; ``r`` accumulates
    iterations, the last update norm and the last Reynolds number reached.
    Each Reynolds number gets at most ``max_newton`` iterations; an update
    norm above ``diverge_factor`` times the first of its Reynolds number, or
    a non-finite one, marks the instance diverged.  ``r.converged`` is set
    when the last Reynolds number reaches ``pseudo_tol``.  Returns the last
    update norm ||dq||/(2N)."""
    cfg = s.cfg
    urot = cfg.u_rot(cfg.t_start)
    res = math.inf
    for k, re in enumerate(ladder):
        last = k == len(ladder) - 1
        tol = pseudo_tol if last else max(pseudo_tol, rung_tol)
        if len(ladder) > 1:
            s.dev.set_re(re)
        r.rungs += 1
        res, first, n = math.inf, None, 0
        while n < max_newton:
            res = s._assemble_and_solve_once(cfg.inv_dtau(), cfg.inv_2dt(), urot)
            n += 1
            r.newton_iters += 1
            r.krylov_iters += s._last_lin.iterations
            r.res = res
            first = res if first is None else first
            if not np.isfinite(res) or res > diverge_factor * first:
                r.diverged = True
                return res
            if res <= tol:
                break
        if not res <= tol:
            return res
        r.re_reached = re
    r.converged = True
    return res


def run_sweep(cases, workers: int = 16, precision: str = "mixed", max_newton: int = 20,
              pseudo_tol: float = 1e-10, krylov_max_it: int = 300,
              diverge_factor: float = 1e3, continuation: float | None = None,
              re_start: float = 80.0, rung_tol: float = 1e-7, **cfg_kw) -> SweepResult:
    """Solve every case to a steady state, ``workers`` instances at a time.

    Each instance runs the steady Newton loop (vorti2d/solver.py:136-145:
    iterate while ||dq||/(2N) > pseudo_tol, at most max_newton times) and
    additionally stops when the update norm exceeds ``diverge_factor`` times
    the first one (a diverging instance), with GMRES capped at
    ``krylov_max_it`` iterations per Newton step.  Handles are created first
    (device allocation synchronises the device, so it is kept out of the
    timed solve phase); ``solve_s`` is the wall time of the concurrent
    solves.

    ``continuation`` (a factor > 1) solves each case above ``re_start`` along
    ``re_ladder``: every Reynolds number but the last to ||dq||/(2N) <=
    ``rung_tol``, starting from the previous one's state, the last to
    ``pseudo_tol``.  Without it every case starts from the free stream at
    its own Re, the reference's steady method."""
    from .solver import Solver
    out = SweepResult(workers=workers)
    t0 = time.perf_counter()
    solvers = [Solver(_config(c, precision, max_newton, pseudo_tol, krylov_max_it, **cfg_kw),
                      mesh=(c.xg, c.yg))
               for c in cases]
    out.setup_s = time.perf_counter() - t0
    results = [None] * len(cases)
    lock = threading.Lock()

    def work(i):
        c, s = cases[i], solvers[i]
        t = time.perf_counter()
        r = CaseResult(c.name, c.re, c.alpha_deg, s.ndof, False, 0, math.inf)
        try:
            solve_case(s, r, re_ladder(c.re, re_start, continuation), max_newton, pseudo_tol,
                       rung_tol, diverge_factor)
            if r.converged:
                fc = s.force_coeffs()
                r.cd, r.cl, r.cm = fc.cd, fc.cl, fc.cm
        except (_lib.V2DError, ValueError) as exc:
            r.error = str(exc)[:200]
        r.seconds = time.perf_counter() - t
        with lock:
            results[i] = r

    t1 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=workers) as pool:
        list(pool.map(work, range(len(cases))))
    out.solve_s = time.perf_counter() - t1
    for s in solvers:
        s.close()
    out.results = results
    return out


def run_sweep_batched(cases, precision: str = "mixed", max_newton: int = 20,
                      pseudo_tol: float = 1e-10, krylov_max_it: int = 300,
                      diverge_factor: float = 1e3, **cfg_kw) -> SweepResult:
    """Solve every case to a steady state in one batch (``v2d_batch_*``).

    Each instance follows the reference's steady loop (vorti2d/solver.py:
    136-145: iterate while ||dq||/(2N) > pseudo_tol, at most max_newton
    times); an instance whose update norm exceeds ``diverge_factor`` times its
    first one, or is not finite, is frozen as diverged.  Every Newton
    iteration of the batch is one iteration of all instances still active.
    ``setup_s`` covers the batch's creation (meshes, metrics, patterns, the
    forest plan, factor storage); ``solve_s`` the Newton iterations."""
    from ctypes import byref, c_void_p
    from .solver import solver_params
    n = len(cases)
    cfgs = [_config(c, precision, max_newton, pseudo_tol, krylov_max_it, **cfg_kw) for c in cases]
    params = (_lib.SolverParams * n)(*[solver_params(c) for c in cfgs])
    xs = [np.asfortranarray(c.xg, dtype=np.float64) for c in cases]
    ys = [np.asfortranarray(c.yg, dtype=np.float64) for c in cases]
    imax = np.array([x.shape[0] for x in xs], dtype=np.intc)
    jmax = np.array([x.shape[1] for x in xs], dtype=np.intc)
    xp = (_lib._dp * n)(*[_lib.dptr(x) for x in xs])
    yp = (_lib._dp * n)(*[_lib.dptr(y) for y in ys])
    out = SweepResult(workers=1, shared_krylov=0)
    t0 = time.perf_counter()
    h = c_void_p()
    _lib.check(_lib.lib().v2d_batch_create(n, _lib.iptr(imax), _lib.iptr(jmax), xp, yp, params,
                                            byref(h)), "batch_create")
    out.setup_s = time.perf_counter() - t0
    results = [CaseResult(c.name, c.re, c.alpha_deg, int(imax[i] * jmax[i]), False, 0, math.inf)
               for i, c in enumerate(cases)]
    active = np.ones(n, dtype=np.intc)
    first = np.full(n, np.nan)
    res = np.zeros(n)
    flags = np.zeros(n, dtype=np.intc)
    try:
        t1 = time.perf_counter()
        for it in range(max_newton):
            st = _lib.LinStats()
            code = _lib.lib().v2d_batch_newton(h, _lib.dptr(res), _lib.iptr(flags), byref(st))
            if code == _lib.V2D_ENONFINITE:
                # instances with a non-finite residual: diverged, frozen; the
                # others are advanced by the next call
                for i in np.nonzero(flags & 6)[0]:
                    results[i].diverged = True
                    results[i].error = "non-finite residual"
                    active[i] = 0
                _lib.check(_lib.lib().v2d_batch_set_active(h, _lib.iptr(active)))
                if not active.any():
                    break
                continue
            if code not in (_lib.V2D_OK, _lib.V2D_ENOTCONVERGED):
                _lib.check(code, "batch_newton")
            out.shared_krylov += st.iterations
            for i in np.nonzero(active)[0]:
                r = results[i]
                r.newton_iters += 1
                r.krylov_iters += st.iterations
                r.res = float(res[i])
                if np.isnan(first[i]):
                    first[i] = res[i]
                if not np.isfinite(res[i]) or res[i] > diverge_factor * first[i]:
                    r.diverged = True
                    active[i] = 0
                elif res[i] <= pseudo_tol:
                    r.converged = True
                    active[i] = 0
            _lib.check(_lib.lib().v2d_batch_set_active(h, _lib.iptr(active)))
            if not active.any():
                break
        out.solve_s = time.perf_counter() - t1
        for i, (c, r) in enumerate(zip(cases, results)):
            r.re_reached = c.re if r.converged else math.nan
            r.rungs = 1
            if r.converged:
                s = c_void_p()
                _lib.check(_lib.lib().v2d_batch_instance(h, i, byref(s)))
                f10 = np.zeros(10)
                rl = -1.0 if c.ref_length is None else float(c.ref_length)
                _lib.check(_lib.lib().v2d_solver_forces(s, float(c.re), rl, 0.0, 0.0,
                                                        _lib.dptr(f10)))
                r.cd, r.cl, r.cm = float(f10[0]), float(f10[1]), float(f10[2])
    finally:
        _lib.lib().v2d_batch_destroy(h)
    out.results = results
    return out
