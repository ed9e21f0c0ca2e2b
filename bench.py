"""Benchmark: unsteady BDF2 dual-time cylinder (181x181 O-grid, Re=100,
dt=0.2, rotational kick 0.5 until t=2, outflow far field, <=5 Newton
iterations per step, GMRES(30)).  The Krylov solve is preconditioned with
the multifrontal LU of each Newton Jacobian: GMRES(30) with 2x2 block Jacobi
does not converge on these pure-Newton (dtau = inf) systems (it stops at the
iteration limit every Newton step), so it would not reproduce the reference's
direct-solve results.

One "step" is one BDF2 physical time step through the device solver.
``value`` = whole-job BDF2 steps/s with the state resident in HBM (headline:
FP32 Krylov inside FP64 Newton / defect correction); the FP64-Krylov form is
measured beside it.  ``e2e`` is the same metric through the public Python API
with the state copied host->device and device->host every step (pinned host
buffers).  ``--impl reference`` times the CPU restatement of the reference
path (C assembly + SuperLU direct solves) on the host cores.

Multi-GPU (``torchrun --nproc-per-node N``): independent replicas, one per
GPU, no collective on the data path; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

IMAX = JMAX = 181
WORKLOAD = dict(re=100.0, steady=False, dt_phys=0.2, rot_speed=0.5, rot_until=2.0,
                farfield_bc="outflow")
SOLVER = dict(ksp_restart=30, ksp_rtol=1e-10, krylov_max_it=3000, pseudo_tol=1e-10,
              max_pseudo_iter=5, precond="lu")
METRIC = "BDF2 steps/s, 181x181 cylinder O-grid Re=100 dt=0.2 (<=5 Newton, GMRES(30))"
WORKLOAD_NAME = "unsteady BDF2 cylinder 181x181 Re=100 dt=0.2 kick 0.5<=2 outflow"
L2_FLUSH_BYTES = 256 << 20
SPMV_BYTES_PER_NNZ = {"fp64": 8 + 4, "fp32": 4 + 4}


# ------------------------------------------------------------------ ranks
def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_dist(world, backend):
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return dist


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- clocks
def _finite_or_none(o):
    if isinstance(o, float):
        return o if math.isfinite(o) else None
    if isinstance(o, dict):
        return {k: _finite_or_none(v) for k, v in o.items()}
    if isinstance(o, (list, tuple)):
        return [_finite_or_none(v) for v in o]
    return o


def jline(obj) -> str:
    """One JSON line; a number that is not finite is written as null (NaN
    and Infinity are not JSON)."""
    return json.dumps(_finite_or_none(obj), allow_nan=False)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed
    region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return self.summary()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return float("nan")
        sm = np.array([num(r[1]) for r in self.rows])
        mx = np.array([num(r[2]) for r in self.rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        sm = sm[np.isfinite(sm)]
        mx = mx[np.isfinite(mx)]
        # fields the driver reports as not available give None, not NaN
        # (NaN is not JSON)
        smax = float(mx.max()) if mx.size else None
        load = sm[sm > 0.5 * smax] if smax is not None else sm
        if not load.size:
            load = sm
        med = float(np.median(load)) if load.size else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(self.rows)}


# ------------------------------------------------------------- our arm
def make_solver(v, xg, yg, precision, lu_reuse=0, lu_steps=0, item_rows=None):
    cfg = v.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                   raise_on_linear_failure=False, precision=precision, lu_reuse_its=lu_reuse,
                   lu_reuse_steps=bool(lu_steps), lu_item_rows=item_rows, **WORKLOAD, **SOLVER)
    return v.Solver(cfg, mesh=(xg, yg))


def flush_l2(torch, buf):
    buf.add_(1.0)


def timed_steps(torch, s, times, k0, K, flush_buf):
    """K BDF2 steps on the solver's stream, each preceded by an L2 flush
    (outside the events), inside the NVTX range v2d_timed (for a profiler's
    launch list of the timed region); returns (per-step ms list, Newton its,
    Krylov its)."""
    import ctypes
    from vorti2d_b200 import _lib
    sp = ctypes.c_void_p()
    _lib.check(_lib.lib().v2d_solver_stream(s.dev.h, ctypes.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    ms, newton, krylov = [], 0, 0
    torch.cuda.nvtx.range_push("v2d_timed")
    for m in range(K):
        flush_l2(torch, flush_buf)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, it, _ = s.advance(times[k0 + m])
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        newton += it
        krylov += s.newton_log[-1][2]
    torch.cuda.nvtx.range_pop()
    return ms, newton, krylov


# Algorithmic bytes per node of the HBM-bound kernels (read inputs + write
# outputs once): metrics x, y -> 10 arrays; assembly 6 metrics + 4 state
# fields -> 23 Jacobian values + 2 right-hand sides (+ 4 block inverses and,
# mixed, an FP32 copy); velocity 5 metrics + psi -> u, v, |V|; SpMV per nnz
# value + column index, plus row pointers and the two vectors.
KERNEL_BYTES = {"metrics": 96, "assemble_fp64": 8 * (6 + 4) + 8 * 23 + 8 * 2 + 8 * 4,
                "assemble_mixed": 8 * (6 + 4) + 12 * 23 + 8 * 2 + 12 * 4, "velocity": 8 * 6 + 8 * 3}


def kernel_rooflines(n_side, hbm_gbs, reps=10):
    """Metrics, assembly, velocity and Krylov SpMV on an n_side x n_side
    cylinder O-grid (state: the far-field initial condition), each timed
    alone after L2 flushes, against the HBM roofline."""
    import ctypes
    import vorti2d_b200 as v
    from vorti2d_b200 import _lib
    xg, yg = v.generate_cylinder(n_side, n_side)
    cfg = v.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                   precond="bjacobi", precision="mixed", **WORKLOAD)
    s = v.Solver(cfg, mesh=(xg, yg))
    N = s.ndof
    nnz = ctypes.c_longlong()
    _lib.check(_lib.lib().v2d_solver_nnz(s.dev.h, ctypes.byref(nnz)))
    out = {}
    for name, which in (("metrics", 0), ("assemble_fp64", 1), ("assemble_mixed", 2),
                        ("velocity", 3)):
        ms = ctypes.c_double()
        _lib.check(_lib.lib().v2d_solver_time_kernel(s.dev.h, which, reps, L2_FLUSH_BYTES,
                                                     ctypes.byref(ms)))
        b = KERNEL_BYTES[name] * N
        out[name] = {"ms": ms.value, "bytes": b, "GBs": b / ms.value / 1e6,
                     "frac": b / ms.value / 1e6 / hbm_gbs}
    _lib.check(_lib.lib().v2d_solver_assemble(s.dev.h, 0.0))
    for prec, fp32 in (("fp64", 0), ("fp32", 1)):
        ms = ctypes.c_double()
        _lib.check(_lib.lib().v2d_solver_time_spmv(s.dev.h, fp32, reps, L2_FLUSH_BYTES,
                                                   ctypes.byref(ms)))
        n = 2 * N
        b = nnz.value * SPMV_BYTES_PER_NNZ[prec] + (n + 1) * 4 + 2 * n * (4 if fp32 else 8)
        out[f"spmv_{prec}"] = {"ms": ms.value, "bytes": b, "GBs": b / ms.value / 1e6,
                               "frac": b / ms.value / 1e6 / hbm_gbs}
    s.close()
    return {"grid": f"{n_side}x{n_side}", "nodes": N, "nnz": nnz.value, "kernels": out}


def run_sweep_workload(args):
    """Batched steady sweep: 96 instances (32 cylinders 129x129, 32 cylinders
    181x181, 32 NACA-0012 257x129; Re ~ U[50,1000], alpha ~ U[-8,8] deg from
    seed 0), steady pure Newton (at most 20 iterations), FP32 Krylov + LU
    inside FP64 defect correction, solved concurrently.  Plain Newton from the
    free stream converges only on part of that Re range, so value = Newton
    iterations per second summed over the instances (the work done), with
    converged solves per second beside it."""
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200.batch import run_sweep, run_sweep_batched, sweep_cases
    torch.cuda.set_device(0)
    cases = sweep_cases(seed=0)
    cont = args.sweep_continuation if args.sweep_continuation > 1.0 else None
    if args.sweep_mode == "batched" and cont is None:
        res = run_sweep_batched(cases, precision=args.sweep_precision,
                                krylov_max_it=args.sweep_krylov_max,
                                diverge_factor=args.sweep_diverge, lu_factors=args.lu_factors)
    else:
        res = run_sweep(cases, workers=args.sweep_workers, precision="mixed", continuation=cont)
    kinds = {}
    for r in res.results:
        k = r.name.rsplit("_", 1)[0]
        d = kinds.setdefault(k, {"instances": 0, "converged": 0, "diverged": 0, "errors": 0,
                                 "newton": 0, "krylov": 0})
        d["instances"] += 1
        d["converged"] += int(r.converged)
        d["diverged"] += int(r.diverged)
        d["errors"] += int(bool(r.error))
        d["newton"] += r.newton_iters
        d["krylov"] += r.krylov_iters
    cpu = None
    if args.cpu_steps > 0:
        from oracle import oracle as O
        sample = [c for c in cases if c.name.startswith("cyl129")][:2]
        t0 = time.perf_counter()
        its = 0
        for c in sample:
            o = O.OracleSolver(c.xg, c.yg, re=c.re, alpha_deg=c.alpha_deg, steady=True,
                               pseudo_tol=1e-10, max_pseudo_iter=5)
            its += o.advance(0.0)[1]
        dt = time.perf_counter() - t0
        cpu = {"value": its / dt, "unit": "Newton iterations/s", "cores": 1, "kind": "port",
               "sample": f"{its} Newton iterations of {len(sample)} 129x129 cylinder instances "
                         "of the sweep, serial (C assembly + SuperLU)"}
    line = {"metric": "Newton iterations/s, 96-instance steady sweep (cylinders 129^2/181^2, "
                      "NACA-0012 257x129)",
            "value": res.newton_per_s, "unit": "Newton iterations/s", "n_gpus": 1,
            "converged_solves_per_s": res.solves_per_s, "newton_iters": res.newton_iters,
            "higher_is_better": True, "dtype": "f32-krylov/f64", "data": "synthetic",
            "config": {"workload": "batched steady sweep, seed 0", "workers": res.workers,
                       "mode": ("one block-diagonal system, one launch per Newton phase"
                                if args.sweep_mode == "batched" and cont is None
                                else "one handle and stream per instance, thread pool"),
                       "precond": "multifrontal LU per Newton iteration",
                       "newton": "<=20 iterations, frozen when ||dq|| > diverge_factor x the first",
                       "krylov_max_it": args.sweep_krylov_max,
                       "precision": args.sweep_precision, "diverge_factor": args.sweep_diverge,
                       "continuation": (f"Re from 80 x{cont} per rung, rungs to ||dq||/(2N) <= 1e-7"
                                        if cont else "none (free stream at the case's Re)")},
            "max_re_converged": max([r.re for r in res.results if r.converged], default=None),
            "min_re_failed": min([r.re for r in res.results if not r.converged], default=None),
            "krylov_iters": res.krylov_iters,
            "errors": sorted({r.error for r in res.results if r.error})[:4],
            "converged": res.converged, "instances": len(cases), "solve_s": res.solve_s,
            "setup_s": res.setup_s, "by_kind": kinds, "cpu_baseline": cpu}
    print(jline(line), flush=True)


def run_adjoint_workload(args):
    """Steady discrete adjoint: NACA-0012 257x193 (256 distinct wall nodes),
    wall displaced by seeded Gaussian bumps of 1e-3 chord, alpha = 4 deg,
    Re = --adjoint-re.  The steady Newton solve (FP64 LU-preconditioned GMRES)
    is timed, then the gradients dCl/dalpha, dCd/dRe and dCd/d(256 wall-normal
    displacements): one FP64 factorization of dR/dq shared by the three
    transposed solves, residual parameter derivatives, and the exact tangent
    derivatives of the residual and the wall forces along all 256 directions.
    value = gradient evaluations (all three) per second.  The steady solve is
    then repeated from the same start on the warm handle, and the line gives
    the time of a gradient set over that of the solve.  --adjoint-dtau > 0
    solves the primal by pseudo-time continuation with switched evolution
    relaxation from that dtau (1/dtau added to the Newton diagonal as the
    reference's dual-time stepping does, dtau growing as the update norm
    falls) where plain Newton from the free stream fails; the adjoint uses
    dR/dq without it."""
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200.adjoint import (deform_ogrid, force_vjp, gaussian_bumps, shape_vjp,
                                      steady_solve_ser)
    torch.cuda.set_device(0)
    base = v.generate_naca0012(257, 193)
    d0 = gaussian_bumps(256, n_bumps=8, amplitude=1e-3, seed=0)
    X, Y = deform_ogrid(*base, d0)
    dtau = args.adjoint_dtau if args.adjoint_dtau > 0 else math.inf
    cfg = v.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                   re=args.adjoint_re, alpha_deg=4.0, steady=True, pseudo_tol=1e-12,
                   max_pseudo_iter=30, ksp_rtol=1e-12,
                   ref_length=1.0, precision="fp64", raise_on_linear_failure=False)
    s = v.Solver(cfg, mesh=(X, Y))
    q0 = s.get_state()

    def primal():
        if math.isinf(dtau):
            return s.advance(0.0)[:2]
        # a second, gentler continuation from the same start if the first
        # fails, then a Reynolds ladder (each rung from the previous state)
        total = 0
        for growth in (2.0, 1.25):
            s.set_state(*q0)
            res, its = steady_solve_ser(s, dtau0=dtau, max_iter=300, growth=growth)
            total += its
            if math.isfinite(res) and res <= cfg.pseudo_tol:
                return res, total
        s.set_state(*q0)
        target = float(cfg.re)
        ladder = (5.0, 10.0, 20.0, 40.0, 70.0, 100.0, 150.0, 200.0, 300.0, 400.0)
        for re_k in [r for r in ladder if r < target] + [target]:
            s.dev.set_re(re_k)
            res, its = steady_solve_ser(s, dtau0=dtau, max_iter=300, growth=1.5, re=re_k)
            total += its
            if not (math.isfinite(res) and res <= cfg.pseudo_tol):
                break
        s.dev.set_re(target)
        return res, total

    t0 = time.perf_counter()
    try:
        res, its = primal()
    except v._lib.V2DError:
        res, its = float("nan"), cfg.max_pseudo_iter
    t_solve = time.perf_counter() - t0
    converged = bool(np.isfinite(res) and res <= cfg.pseudo_tol)
    line = {"metric": "steady adjoint gradients/s (dCl/dalpha, dCd/dRe, dCd/d(256 wall "
                      "displacements)), NACA-0012 257x193",
            "unit": "gradient sets/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "steady discrete adjoint, NACA-0012 257x193, alpha 4 deg, "
                                   f"Re {args.adjoint_re:g}, 8 seeded 1e-3-chord wall bumps",
                       "primal": "plain Newton" if math.isinf(dtau)
                                 else f"pseudo-time continuation (SER) from dtau {dtau:g}"},
            "steady_newton_its": its, "steady_res": res, "steady_converged": converged,
            "steady_solve_s": t_solve}
    if not converged:
        line.update(value=None, note="the primal did not converge from the free stream at "
                                     "this Re; no gradient at an unconverged state")
        print(jline(line), flush=True)
        s.close()
        return
    reps = max(1, args.steps // 5)
    t0 = time.perf_counter()
    for _ in range(reps):
        d_alpha, _, info = force_vjp(s, (1.0, 0.0, 0.0))
        _, d_re, _ = force_vjp(s, (0.0, 1.0, 0.0))
        gshape, sinfo = shape_vjp(s, (0.0, 1.0, 0.0), base)
    dt = (time.perf_counter() - t0) / reps
    # the primal again from the same free-stream start, now that plan, factor
    # storage and graphs exist: the cost a gradient set is compared with
    s.set_state(*q0)
    t0 = time.perf_counter()
    try:
        primal()
        t_warm = time.perf_counter() - t0
    except v._lib.V2DError:
        t_warm = float("nan")
    line.update(steady_solve_warm_s=t_warm, gradient_set_over_primal=dt / t_warm)
    line.update(value=1.0 / dt, ms_per_gradient_set=1e3 * dt, reps=reps,
                dCl_dalpha=d_alpha, dCd_dRe=d_re, dCd_dd_norm=float(np.linalg.norm(gshape)),
                adjoint_refinements=sinfo["refinements"], adjoint_rel_res=sinfo["rel_res"])
    print(jline(line), flush=True)
    s.close()


def fp64_gemm_tflops(torch, n=8192, reps=5):
    """Dense FP64 GEMM rate of this GPU (torch.matmul, i.e. the vendor BLAS,
    n x n x n), CUDA events: the reference rate for the factorization's
    FP64 contractions."""
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = torch.matmul(a, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.matmul(a, b, out=c)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, b, c
    return 2.0 * n ** 3 / (ms * 1e-3) / 1e12


def factor_rate(torch, _lib, s):
    """One LU factorization of the handle's current matrix, timed per launch
    (v2d_solver_time_lu_factor), its flops (v2d_solver_lu_stats) and the
    rate against the FP64 GEMM rate of the same GPU, with the time per
    kernel kind."""
    import ctypes
    st = (ctypes.c_double * 6)()
    _lib.check(_lib.lib().v2d_solver_lu_stats(s.dev.h, st))
    cap = 16384
    ms = (ctypes.c_double * cap)()
    codes = (ctypes.c_int * cap)()
    n = ctypes.c_int()
    _lib.check(_lib.lib().v2d_solver_time_lu_factor(s.dev.h, 1, ms, codes, cap, ctypes.byref(n)))
    fkinds = ["rowscale", "scatter", "extend_add", "panel", "l21_swap_trsm", "-", "gemm", "trinv",
              "trcopy", "gh", "ghcopy", "round_f32"]
    by_kind = {}
    for k in range(n.value):
        kind = fkinds[codes[k] // 1000]
        by_kind[kind] = by_kind.get(kind, 0.0) + ms[k]
    total = sum(ms[k] for k in range(n.value))
    tf = st[3] / (total * 1e-3) / 1e12
    peak = fp64_gemm_tflops(torch)
    return {"ms": total, "launches": n.value, "flops": st[3], "tflops": tf,
            "fp64_gemm_tflops": peak, "frac_of_fp64_gemm": tf / peak,
            "fronts": int(st[0]), "levels": int(st[1]), "factor_entries": st[2],
            "by_kind_ms": {k: round(v, 3) for k, v in by_kind.items()}}


def run_large_workload(args):
    """Large unsteady run: cylinder O-grid N x N (default 2049, 8.4M
    unknowns), Re 200, dt 0.05, outflow far field, BDF2 with at most 5 Newton
    iterations per step, FP64 LU + Krylov by default (FP32 factors with
    pivoting inside 32-row blocks do not precondition these fronts well
    enough).  One warm-up step (plan, factors and graphs), then --large-steps timed
    steps with CUDA events; the LU solve of one GMRES iteration is timed
    after an L2 flush against the HBM roofline (at this size the factors do
    not fit in L2)."""
    import ctypes
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200 import _lib
    torch.cuda.set_device(0)
    n = args.large_grid
    xg, yg = v.generate_cylinder(n, n)
    cfg = v.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                   re=200.0, steady=False, dt_phys=0.05, farfield_bc="outflow",
                   raise_on_linear_failure=False, precision=args.large_precision,
                   lu_reuse_its=args.large_reuse, lu_reuse_steps=bool(args.lu_reuse_steps),
                   **SOLVER)
    t0 = time.perf_counter()
    s = v.Solver(cfg, mesh=(xg, yg))
    setup_s = time.perf_counter() - t0
    times = s.times()
    t0 = time.perf_counter()
    s.advance(times[0])
    torch.cuda.synchronize()
    first_s = time.perf_counter() - t0
    tuning = None
    if args.lu_tune and SOLVER.get("lu_solve", "flow") == "flow":
        from vorti2d_b200.tune import tune_lu_solve
        t0 = time.perf_counter()
        tuning = tune_lu_solve(s, sweeps=1)
        tuning["seconds"] = time.perf_counter() - t0
    phase_times(_lib, s, reset=True)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    K = args.large_steps
    ms, newton, krylov = timed_steps(torch, s, times, 1, K, flush)
    ph = phase_times(_lib, s)
    lu_ms = ctypes.c_double()
    fb = ctypes.c_longlong()
    _lib.check(_lib.lib().v2d_solver_time_lu_apply(s.dev.h, 3, L2_FLUSH_BYTES,
                                                  ctypes.byref(lu_ms), ctypes.byref(fb)))
    factor = factor_rate(torch, _lib, s)
    hbm = 6650.0
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            hbm = json.load(fh)["hbm_gbs"]
    except (OSError, ValueError, KeyError):
        pass
    gbs = fb.value / (lu_ms.value * 1e-3) / 1e9
    step_ms = float(np.mean(ms))
    line = {"metric": f"BDF2 steps/s, {n}x{n} cylinder O-grid Re=200 dt=0.05 (<=5 Newton, "
                      "GMRES(30))",
            "value": 1e3 / step_ms, "unit": "steps/s", "n_gpus": 1, "steps": K, "warmup": 1,
            "ms_per_step": step_ms, "higher_is_better": True,
            "dtype": "f32-krylov/f64" if args.large_precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": f"large unsteady BDF2 cylinder {n}x{n} Re=200 dt=0.05 outflow",
                       "unknowns": 2 * n * n, "lu_reuse_its": args.large_reuse,
                       "lu_factors": SOLVER.get("lu_factors"),
                       "lu_reuse_steps": args.lu_reuse_steps,
                       "l2": "flushed (256 MiB write) before every timed step"},
            "setup_s": setup_s, "first_step_s": first_s, "newton_per_step": newton / K,
            "krylov_per_step": krylov / K,
            "ms_per_newton": {"assembly": ph[0] / max(ph[4], 1), "factor": ph[1] / max(ph[4], 1),
                              "krylov": ph[2] / max(ph[4], 1), "update": ph[3] / max(ph[4], 1)},
            "factorizations_per_step": ph[5] / K,
            "roofline": {"bound": "hbm", "kernel": "lu_apply_" + ("fp32" if args.large_precision
                                                                 == "mixed" else "fp64"),
                         "achieved": gbs,
                         "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "bytes_per_launch": fb.value, "ms_per_launch": lu_ms.value},
            "factorization": factor, "lu_tuning": tuning,
            "cd": s.force_coeffs().cd}
    print(jline(line), flush=True)
    s.close()


def run_unsteady_adjoint_workload(args):
    """Unsteady discrete adjoint: time-mean Cd over --ua-steps BDF2 steps of
    the cylinder N x N (default 181), Re 200, dt 0.05, outflow far field,
    every step converged to 1e-12, and its gradient with respect to (alpha,
    Re) with a checkpoint every --ua-checkpoint steps (forward run, then per
    segment: recomputation from the checkpoint and a backward sweep of FP64
    transposed solves).  value = gradients per second (wall clock of the
    whole forward + backward computation)."""
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200.unsteady_adjoint import unsteady_mean_force_vjp
    torch.cuda.set_device(0)
    n = args.ua_grid
    mesh = v.generate_cylinder(n, n)

    def make():
        cfg = v.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                       re=200.0, steady=False, dt_phys=0.05, farfield_bc="outflow",
                       pseudo_tol=1e-12, max_pseudo_iter=20, ksp_rtol=1e-12,
                       precision="fp64", raise_on_linear_failure=False,
                       lu_reuse_its=args.ua_reuse, lu_reuse_steps=args.ua_reuse > 0)
        return v.Solver(cfg, mesh=mesh)

    unsteady_mean_force_vjp(make, 2, (0.0, 1.0, 0.0), checkpoint_every=1)   # warm-up
    torch.cuda.synchronize()
    # device memory in use, sampled once a second during the run (the
    # library's own allocations are not torch's, so ask the driver)
    peak = [0]
    done = threading.Event()

    def watch():
        while not done.is_set():
            free, total = torch.cuda.mem_get_info()
            peak[0] = max(peak[0], total - free)
            done.wait(1.0)

    th = threading.Thread(target=watch, daemon=True)
    th.start()
    t0 = time.perf_counter()
    J, d_alpha, d_re, info = unsteady_mean_force_vjp(make, args.ua_steps, (0.0, 1.0, 0.0),
                                                     checkpoint_every=args.ua_checkpoint)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    done.set()
    th.join()
    line = {"metric": f"unsteady adjoint gradients/s (mean Cd over {args.ua_steps} BDF2 steps, "
                      f"d/dalpha and d/dRe), {n}x{n} cylinder Re=200 dt=0.05",
            "value": 1.0 / dt, "unit": "gradients/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"unsteady discrete adjoint, cylinder {n}x{n}, "
                                   f"{args.ua_steps} steps, checkpoint every "
                                   f"{args.ua_checkpoint}",
                       "lu_reuse_its": args.ua_reuse},
            "seconds": dt, "mean_cd": J, "dJ_dalpha": d_alpha, "dJ_dRe": d_re,
            "device_memory_peak_gb": peak[0] / 1e9, **info}
    print(jline(line), flush=True)


def phase_times(_lib, s, reset=False):
    """(assembly, factorization, Krylov, update) device ms summed over Newton
    iterations, and the iteration count."""
    import ctypes
    out = (ctypes.c_double * 6)()
    _lib.check(_lib.lib().v2d_solver_phase_times(s.dev.h, out, int(reset)))
    return list(out)


def profile_newton(args):
    """One warm-up BDF2 step of the workload (captures the CUDA graphs), then
    exactly one Newton iteration inside the NVTX range "v2d_newton"; for
    `ncu --nvtx --nvtx-include v2d_newton/` launch lists of one iteration."""
    import torch
    import vorti2d_b200 as v
    torch.cuda.set_device(0)
    xg, yg = v.generate_cylinder(IMAX, JMAX)
    prec = "mixed" if args.precision == "both" else args.precision
    s = make_solver(v, xg, yg, prec)
    times = s.times()
    s.advance(times[0])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("v2d_newton")
    code, res, lin = s.dev.newton(s.cfg.u_rot(times[1]))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(jline({"profile": "one Newton iteration", "precision": prec, "code": code,
                      "res": res, "krylov_its": lin.iterations}), flush=True)
    s.close()


def profile_lu_apply(args):
    """Two steps of the workload (factors, graphs), the autotuned work-item
    split, then two warm LU preconditioner solves inside the NVTX range
    v2d_lu_apply (for a profiler capture of the dataflow solve kernel)."""
    import ctypes
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200 import _lib
    from vorti2d_b200.tune import tune_lu_solve
    torch.cuda.set_device(0)
    xg, yg = v.generate_cylinder(IMAX, JMAX)
    prec = "mixed" if args.precision == "both" else args.precision
    s = make_solver(v, xg, yg, prec, args.lu_reuse, args.lu_reuse_steps)
    times = s.times()
    for m in range(2):
        s.advance(times[m])
    rec = tune_lu_solve(s) if args.lu_tune else None
    torch.cuda.synchronize()
    ms, fb = ctypes.c_double(), ctypes.c_longlong()
    torch.cuda.nvtx.range_push("v2d_lu_apply")
    _lib.check(_lib.lib().v2d_solver_time_lu_apply(s.dev.h, 2, 0, ctypes.byref(ms),
                                                   ctypes.byref(fb)))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(jline({"profile": "LU apply", "precision": prec, "ms": ms.value,
                      "factor_bytes": fb.value, "tuning": rec}), flush=True)
    s.close()


def profile_lu_factor(args):
    """Two steps of the workload on the cylinder --profile-grid, then one LU
    factorization of the current Jacobian inside the NVTX range v2d_lu_factor
    (for a profiler capture of one factorization kernel)."""
    import ctypes
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200 import _lib
    torch.cuda.set_device(0)
    grid = args.profile_grid
    xg, yg = v.generate_cylinder(grid, grid)
    prec = "mixed" if args.precision == "both" else args.precision
    s = make_solver(v, xg, yg, prec, args.lu_reuse, args.lu_reuse_steps)
    times = s.times()
    for m in range(2):
        s.advance(times[m])
    torch.cuda.synchronize()
    cap = 16384
    ms = (ctypes.c_double * cap)()
    codes = (ctypes.c_int * cap)()
    n = ctypes.c_int()
    torch.cuda.nvtx.range_push("v2d_lu_factor")
    _lib.check(_lib.lib().v2d_solver_time_lu_factor(s.dev.h, 1, ms, codes, cap, ctypes.byref(n)))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(jline({"profile": "LU factorization", "grid": f"{grid}x{grid}", "precision": prec,
                      "ms": sum(ms[k] for k in range(n.value)), "launches": n.value}), flush=True)
    s.close()


def profile_lu_launches(args):
    """Per-launch device time of one LU preconditioner solve after two steps
    of the workload, with the factors warm in L2 (as inside GMRES) and after
    an L2 flush."""
    import ctypes
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200 import _lib
    torch.cuda.set_device(0)
    grid = args.profile_grid
    xg, yg = v.generate_cylinder(grid, grid)
    prec = "mixed" if args.precision == "both" else args.precision
    s = make_solver(v, xg, yg, prec, args.lu_reuse, args.lu_reuse_steps)
    times = s.times()
    for m in range(2):
        s.advance(times[m])
    kinds = ["forward_level", "backward_level", "dataflow"]
    out = {"profile": "LU solve launches", "precision": prec, "grid": f"{grid}x{grid}",
           "lu_factors": SOLVER.get("lu_factors", "fp32")}
    if args.lu_tune and SOLVER.get("lu_solve", "flow") == "flow":
        from vorti2d_b200.tune import tune_lu_solve
        out["lu_tuning"] = tune_lu_solve(s, sweeps=1 if grid > 513 else 2)
    for label, flush in (("warm", 0), ("cold", L2_FLUSH_BYTES)):
        cap = 256
        ms = (ctypes.c_double * cap)()
        codes = (ctypes.c_int * cap)()
        n = ctypes.c_int()
        _lib.check(_lib.lib().v2d_solver_time_lu_launches(s.dev.h, 20 if grid <= 513 else 3,
                                                         flush, ms, codes, cap,
                                                         ctypes.byref(n)))
        rows = [(kinds[codes[k] // 1000], codes[k] % 1000, ms[k]) for k in range(n.value)]
        by_kind = {}
        for kind, _, t in rows:
            by_kind[kind] = by_kind.get(kind, 0.0) + t
        out[label] = {"total_ms": sum(t for _, _, t in rows), "launches": len(rows),
                      "by_kind_ms": by_kind,
                      "per_launch_us": [[kind, lvl, round(1e3 * t, 2)] for kind, lvl, t in rows]}
    if SOLVER.get("lu_solve", "flow") == "flow":
        out["dataflow_trace"] = lu_trace_summary(s)
    fkinds = ["rowscale", "scatter", "extend_add", "panel", "l21_swap_trsm", "-", "gemm", "trinv",
              "trcopy", "gh", "ghcopy", "round_f32"]
    cap = 16384
    ms = (ctypes.c_double * cap)()
    codes = (ctypes.c_int * cap)()
    n = ctypes.c_int()
    _lib.check(_lib.lib().v2d_solver_time_lu_factor(s.dev.h, 5 if grid <= 513 else 2, ms, codes,
                                                    cap, ctypes.byref(n)))
    by_kind, by_level, by_level_kind = {}, {}, {}
    for k in range(n.value):
        kind, lvl = fkinds[codes[k] // 1000], codes[k] % 1000
        by_kind[kind] = by_kind.get(kind, 0.0) + ms[k]
        by_level[lvl] = by_level.get(lvl, 0.0) + ms[k]
        row = by_level_kind.setdefault(lvl, {})
        row[kind] = round(row.get(kind, 0.0) + 1e3 * ms[k], 1)
    st = (ctypes.c_double * 6)()
    _lib.check(_lib.lib().v2d_solver_lu_stats(s.dev.h, st))
    total = sum(ms[k] for k in range(n.value))
    top = int(st[1]) - 2   # the two top levels launch by launch
    out["factor"] = {"total_ms": total, "launches": n.value, "flops": st[3],
                     "tflops": st[3] / (total * 1e-3) / 1e12,
                     "by_kind_ms": by_kind, "by_level_ms": by_level,
                     "by_level_kind_us": by_level_kind,
                     "top_levels_us": [[fkinds[codes[k] // 1000], codes[k] % 1000,
                                        round(1e3 * ms[k], 1)]
                                       for k in range(n.value) if codes[k] % 1000 >= top]}
    print(jline(out), flush=True)
    s.close()


def lu_trace_summary(s):
    """Per level and sweep of one dataflow LU solve (v2d_solver_trace_lu_apply):
    items, the time from the solve's start to the level's first item start
    and last item end, the mean time an item runs and the mean time it
    waited for its dependencies (us)."""
    import ctypes
    from vorti2d_b200 import _lib
    cap = 1 << 20
    ticks = np.zeros(3 * cap, dtype=np.uint64)
    items = np.zeros(12 * cap, dtype=np.intc)
    n = ctypes.c_int()
    _lib.check(_lib.lib().v2d_solver_trace_lu_apply(
        s.dev.h, ticks.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)), _lib.iptr(items), cap,
        ctypes.byref(n)))
    n = n.value
    t = ticks[:3 * n].reshape(n, 3).astype(np.float64) * 1e-3
    it = items[:12 * n].reshape(n, 12)
    t -= t[:, 0].min()
    levels = []
    for sweep in (0, 1):
        for L in sorted(set(it[it[:, 0] == sweep, 10].tolist()), reverse=bool(sweep)):
            sel = (it[:, 0] == sweep) & (it[:, 10] == L)
            levels.append({"sweep": ["fwd", "bwd"][sweep], "level": int(L),
                           "items": int(sel.sum()),
                           "first_start_us": round(float(t[sel, 0].min()), 2),
                           "last_end_us": round(float(t[sel, 2].max()), 2),
                           "mean_run_us": round(float(np.mean(t[sel, 2] - t[sel, 1])), 2),
                           "mean_wait_us": round(float(np.mean(t[sel, 1] - t[sel, 0])), 2)})
    return {"total_us": round(float(t[:, 2].max()), 2), "items": n, "levels": levels}


def run_ours(args, rank, world, local_rank):
    import torch
    import vorti2d_b200 as v
    from vorti2d_b200 import _lib
    torch.cuda.set_device(local_rank)
    xg, yg = v.generate_cylinder(IMAX, JMAX)
    flush_buf = torch.zeros(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    K, W = args.steps, args.warmup
    results = {}
    legs = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    launches = {}
    for prec in legs:
        s = make_solver(v, xg, yg, prec, args.lu_reuse, args.lu_reuse_steps)
        times = s.times()
        for m in range(W):
            s.advance(times[m])
            if m == 0 and args.lu_tune:
                # work-item split of the LU solve, tuned on this solver's
                # factors after the first warm-up step (the remaining ones
                # capture the GMRES graphs with the chosen split)
                from vorti2d_b200.tune import tune_lu_solve
                results.setdefault("lu_tuning", {})[prec] = tune_lu_solve(s)
        barrier(world)
        torch.cuda.synchronize()
        clocks = ClockSampler(local_rank).start() if prec == legs[0] else None
        phase_times(_lib, s, reset=True)
        c0 = _lib.lib().v2d_launch_count()
        t0 = time.perf_counter()
        ms, nit, kit = timed_steps(torch, s, times, W, K, flush_buf)
        wall = time.perf_counter() - t0
        c1 = _lib.lib().v2d_launch_count()
        ph = phase_times(_lib, s)
        if clocks is not None:
            results["clocks"] = clocks.stop()
        torch.cuda.synchronize()
        barrier(world)
        tot_ms = max_over_ranks(sum(ms), world, "cuda")
        fc = s.force_coeffs()
        nn = max(ph[4], 1.0)
        results[prec] = dict(ms_per_step=tot_ms / K, newton=nit / K, krylov=kit / K,
                             cd=fc.cd, cl=fc.cl, wall_s=wall, t_end=times[W + K - 1],
                             ms_per_newton={"assembly": ph[0] / nn, "factor": ph[1] / nn,
                                            "krylov": ph[2] / nn, "update": ph[3] / nn},
                             factorizations_per_step=ph[5] / K)
        launches[prec] = c1 - c0
        if prec == legs[0]:
            # dominant unit: the LU preconditioner solve of a GMRES iteration,
            # timed alone after L2 flushes; the Krylov SpMV beside it
            import ctypes
            ms_lu, fb = ctypes.c_double(), ctypes.c_longlong()
            _lib.check(_lib.lib().v2d_solver_time_lu_apply(s.dev.h, 20, L2_FLUSH_BYTES,
                                                           ctypes.byref(ms_lu), ctypes.byref(fb)))
            results["lu_apply_ms"], results["lu_factor_bytes"] = ms_lu.value, fb.value
            ms_spmv = _spmv_time(_lib, s, fp32=(prec == "mixed"))
            results["spmv_ms"] = ms_spmv
            import ctypes
            nnz = ctypes.c_longlong()
            _lib.check(_lib.lib().v2d_solver_nnz(s.dev.h, ctypes.byref(nnz)))
            results["nnz"] = nnz.value
            # e2e: the same steps again through the public API, with the
            # state copied host->device and back every step
            rows = results.get("lu_tuning", {}).get(prec, {}).get("rows")
            s2 = make_solver(v, xg, yg, prec, args.lu_reuse, args.lu_reuse_steps, rows)
            for m in range(W):
                s2.advance(times[m])
            results["e2e"] = _e2e(torch, v, s2, times, W, K, flush_buf)
            s2.close()
        s.close()
    return results, launches


def _spmv_time(_lib, s, fp32, reps=20):
    import ctypes
    out = ctypes.c_double()
    _lib.check(_lib.lib().v2d_solver_time_spmv(s.dev.h, int(fp32), reps, L2_FLUSH_BYTES,
                                               ctypes.byref(out)))
    return out.value


def _e2e(torch, v, s, times, k0, K, flush_buf):
    """Steps k0 .. k0+K-1 (the timed steps of the device-resident leg) through
    Solver.set_state / advance / state readback with pinned host buffers; the
    copies are inside the timed region, the L2 flush before each step is not."""
    N = s.ndof
    host = [torch.empty(N, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
    s.get_state(out=host)
    dt = 0.0
    for m in range(K):
        flush_l2(torch, flush_buf)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.set_state(*host)
        s.advance(times[k0 + m])
        s.get_state(out=host)
        dt += time.perf_counter() - t0
    return dict(steps_per_s=K / dt, h2d=4 * N * 8, d2h=4 * N * 8, steps=K)


# ------------------------------------------------------------ CPU arm
def _oracle_solver():
    from oracle import oracle as O
    xg, yg = O.generate_cylinder(IMAX, JMAX)
    return O, O.OracleSolver(xg, yg, pseudo_tol=SOLVER["pseudo_tol"],
                             max_pseudo_iter=SOLVER["max_pseudo_iter"], **WORKLOAD)


def _cpu_replica(warmup, steps, barrier, queue):
    """One replica of the CPU restatement: `warmup` untimed steps from t=0,
    then `steps` timed ones (the same window as the device's timed steps)."""
    _, s = _oracle_solver()
    times = s.times()
    for m in range(warmup):
        s.advance(times[m])
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for m in range(warmup, warmup + steps):
        s.advance(times[m])
    dt = time.perf_counter() - t0
    if queue is not None:
        queue.put(dt)
    return dt


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_cpu_reference(steps, warmup=0, procs=1):
    """CPU restatement of the reference path (C assembly restating
    vorti2d_core.f90 + SuperLU direct solves standing in for MUMPS), one
    single-threaded replica per process like one reference rank each.
    `procs` replicas (spawned processes, one BLAS thread each) run the same
    steps at once, timed over the same window; returns (whole-job steps/s,
    mean steps/s of one replica, slowest replica's seconds)."""
    if procs <= 1:
        dt = _cpu_replica(warmup, steps, None, None)
        return steps / dt, steps / dt, dt
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier, queue = ctx.Barrier(procs), ctx.Queue()
    saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                             "MKL_NUM_THREADS")}
    for k in saved:
        os.environ[k] = "1"
    try:
        ps = [ctx.Process(target=_cpu_replica, args=(warmup, steps, barrier, queue))
              for _ in range(procs)]
        for p in ps:
            p.start()
        dts = [queue.get() for _ in ps]
        for p in ps:
            p.join()
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    slow = max(dts)
    return procs * steps / slow, float(np.mean([steps / d for d in dts])), slow


def cpu_iterative_sample(warmup):
    """The reference's iterative CPU solve (gmres_asm) against its direct one
    on the same system: after `warmup` steps from t=0, the first Newton
    Jacobian of the next step solved by SuperLU and by GMRES(200) with a
    threshold ILU (scipy), one core each."""
    import scipy.sparse.linalg as spla
    O, s = _oracle_solver()
    times = s.times()
    for m in range(warmup):
        s.advance(times[m])
    t = times[warmup]
    ci, cj, cv, nnz, b = s.assemble(O.u_rot(t, s.steady, s.rot_speed, s.rot_until))
    A = O.canonical_csr(ci[:nnz], cj[:nnz], cv[:nnz], 2 * s.ndof, 2 * s.ndof)
    t0 = time.perf_counter()
    x = spla.spsolve(A.tocsc(), b)
    t_lu = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, its, conv, rel = O.gmres_ilu_solve(A, b, rtol=SOLVER["ksp_rtol"])
    t_it = time.perf_counter() - t0
    return {"system": f"first Newton Jacobian of step {warmup} (t={t:.1f})",
            "superlu_s": t_lu,
            "gmres_ilu": {"s": t_it, "iterations": its, "converged": bool(conv),
                          "rel_residual": rel,
                          "solver": "GMRES(200), rtol 1e-10, at most 2000 iterations, "
                                    "scipy spilu (ILUTP, drop 1e-3, fill 10, diagonal "
                                    "pivots) standing in for PETSc ASM/ILU(1)"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"])
    ap.add_argument("--cpu-steps", type=int, default=2,
                    help="timed steps of the one-core CPU sample in the device arm's line")
    ap.add_argument("--cpu-procs", type=int, default=128,
                    help="--impl reference: at most this many CPU replicas (one per core)")
    ap.add_argument("--lu-reuse", type=int, default=8,
                    help="keep LU factors while GMRES needs at most this many iterations "
                         "(0: factor every Newton Jacobian)")
    ap.add_argument("--lu-factors", default="fp32", choices=["fp32", "fp64"],
                    help="mixed leg: LU factorization in FP32, or in FP64 rounded to FP32 "
                         "for the FP32 solve")
    ap.add_argument("--lu-tune", type=int, default=1, choices=[0, 1],
                    help="tune the LU solve's work-item split on the warmed-up solver before "
                         "timing (vorti2d_b200.tune)")
    ap.add_argument("--lu-solve", default="flow", choices=["flow", "levels"],
                    help="LU preconditioner solve: one dataflow launch over the front tree "
                         "(flow) or one launch per level and sweep (levels)")
    ap.add_argument("--lu-reuse-steps", type=int, default=1, choices=[0, 1],
                    help="1: keep the LU factors across time steps (and the e2e leg's "
                         "set_state) under the same rule; 0: refactor at every step")
    ap.add_argument("--kernels-grid", type=int, default=2049,
                    help="grid side of the HBM-bound kernel roofline table (0: skip)")
    ap.add_argument("--workload", default="unsteady", choices=["unsteady", "sweep", "adjoint", "large",
                                                    "unsteady_adjoint"],
                    help="unsteady: the BDF2 benchmark; sweep: the batched steady sweep; "
                         "adjoint: steady adjoint gradients; large: the large unsteady grid; "
                         "unsteady_adjoint: the checkpointed unsteady adjoint")
    ap.add_argument("--sweep-workers", type=int, default=16)
    ap.add_argument("--sweep-precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--sweep-krylov-max", type=int, default=300,
                    help="sweep: GMRES iterations per Newton step at most")
    ap.add_argument("--sweep-diverge", type=float, default=1e3,
                    help="sweep: an instance whose update norm exceeds this factor times its "
                         "first is frozen as diverged")
    ap.add_argument("--sweep-mode", default="batched", choices=["batched", "streams"],
                    help="sweep: all instances as one block-diagonal system (batched) or one "
                         "handle and stream per instance")
    ap.add_argument("--sweep-continuation", type=float, default=0.0,
                    help="sweep: Reynolds continuation factor per rung from Re 80 (0: none, "
                         "plain Newton from the free stream as the reference)")
    ap.add_argument("--large-grid", type=int, default=2049,
                    help="grid side of the large unsteady workload (--workload large)")
    ap.add_argument("--large-reuse", type=int, default=12,
                    help="large: keep the (expensive) FP64 factors while GMRES needs at most "
                         "this many iterations")
    ap.add_argument("--large-steps", type=int, default=3,
                    help="timed BDF2 steps of the large unsteady workload")
    ap.add_argument("--large-precision", default="fp64", choices=["mixed", "fp64"],
                    help="LU factors and Krylov vectors of the large unsteady workload")
    ap.add_argument("--ua-grid", type=int, default=181,
                    help="grid side of the unsteady adjoint workload")
    ap.add_argument("--ua-steps", type=int, default=20,
                    help="BDF2 steps of the unsteady adjoint workload")
    ap.add_argument("--ua-reuse", type=int, default=0,
                    help="unsteady adjoint: keep the forward solve's LU factors across Newton "
                         "iterations and steps while GMRES needs at most this many iterations")
    ap.add_argument("--ua-checkpoint", type=int, default=5,
                    help="checkpoint spacing of the unsteady adjoint workload")
    ap.add_argument("--adjoint-dtau", type=float, default=0.0,
                    help="adjoint workload: pseudo-time step of the steady primal (0: plain "
                         "Newton, dtau = inf)")
    ap.add_argument("--adjoint-re", type=float, default=500.0,
                    help="Reynolds number of the adjoint workload (--workload adjoint)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="print only the HBM-bound kernel roofline table (--kernels-grid)")
    ap.add_argument("--lu-apply-profile", action="store_true",
                    help="two steps, then two warm LU solves in the NVTX range v2d_lu_apply")
    ap.add_argument("--profile-grid", type=int, default=IMAX,
                    help="grid of the --lu-launches profile (the cylinder O-grid N x N)")
    ap.add_argument("--lu-factor-profile", action="store_true",
                    help="one LU factorization inside the NVTX range v2d_lu_factor (profiling)")
    ap.add_argument("--lu-launches", action="store_true",
                    help="per-launch device time of one LU preconditioner solve, warm and cold")
    ap.add_argument("--profile-newton", action="store_true",
                    help="one warm-up step, then one Newton iteration in NVTX range v2d_newton")
    args = ap.parse_args()
    SOLVER["lu_solve"] = args.lu_solve
    SOLVER["lu_factors"] = args.lu_factors
    rank, world, local_rank = dist_env()
    if args.profile_newton:
        profile_newton(args)
        return
    if args.lu_launches:
        profile_lu_launches(args)
        return
    if args.lu_apply_profile:
        profile_lu_apply(args)
        return
    if args.lu_factor_profile:
        profile_lu_factor(args)
        return
    if args.workload == "sweep" and args.impl == "ours":
        run_sweep_workload(args)
        return
    if args.workload == "adjoint" and args.impl == "ours":
        run_adjoint_workload(args)
        return
    if args.workload == "large" and args.impl == "ours":
        run_large_workload(args)
        return
    if args.workload == "unsteady_adjoint" and args.impl == "ours":
        run_unsteady_adjoint_workload(args)
        return
    if args.kernels_only:
        import torch
        torch.cuda.set_device(0)
        hbm = 6650.0
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
                hbm = json.load(fh)["hbm_gbs"]
        except (OSError, ValueError, KeyError):
            pass
        print(jline(kernel_rooflines(args.kernels_grid, hbm, reps=3)), flush=True)
        return

    if args.impl == "reference":
        # CPU restatement on rank 0 only; other ranks exit without work
        if rank != 0:
            return
        # the device arm's window (W untimed steps from t=0, then K timed
        # ones), on one replica per host core; a CPU step takes seconds, so K
        # is capped to keep the run within a few minutes
        K = max(1, min(args.steps, 20))
        W = args.warmup
        P = max(1, min(host_cores(), args.cpu_procs))
        val, per_rep, dt = run_cpu_reference(K, W, P)
        it_sample = cpu_iterative_sample(W)
        line = {
            "metric": METRIC, "value": val, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": 1e3 * dt / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD_NAME,
                       "solver": "C restatement of vorti2d_core.f90 + scipy SuperLU "
                                 "(MUMPS stand-in), one replica per core",
                       "replicas": P},
            "cpu_baseline": {"value": val, "unit": "steps/s", "cores": P, "kind": "port",
                             "sample": f"steps {W}..{W + K - 1} (t={0.2 * W:.1f}..."
                                       f"{0.2 * (W + K - 1):.1f}) of the workload, the "
                                       f"device arm's timed window, on {P} independent "
                                       "replicas at once (whole-job steps/s)",
                             "per_replica_steps_per_s": per_rep,
                             "linear_solve_sample": it_sample},
            "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(jline(line), flush=True)
        return

    init_dist(world, "nccl")
    res, launches = run_ours(args, rank, world, local_rank)
    head = "mixed" if "mixed" in res else args.precision
    ms_head = res[head]["ms_per_step"]
    value = world * 1000.0 / ms_head
    if rank != 0:
        return
    cpu = None
    if world == 1 and args.cpu_steps > 0:
        W = args.warmup
        cval, _, _ = run_cpu_reference(args.cpu_steps, W, 1)
        cpu = {"value": cval, "unit": "steps/s", "cores": 1, "kind": "port",
               "sample": f"steps {W}..{W + args.cpu_steps - 1} of the same workload (the "
                         "first of the device's timed steps; C assembly + SuperLU, one core); "
                         "bench.py --impl reference runs the whole window on every core"}
    nnz = res["nnz"]
    n = 2 * IMAX * JMAX
    prec_key = "fp32" if head == "mixed" else "fp64"
    bytes_spmv = nnz * SPMV_BYTES_PER_NNZ[prec_key] + (n + 1) * 4 + 2 * n * (4 if prec_key == "fp32" else 8)
    peaks, peak_src = {"hbm_gbs": 6650.0}, "fallback 6.65 TB/s (no measured peaks file)"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks, peak_src = json.load(fh), "measured hbm_gbs"
    except (OSError, ValueError):
        pass
    achieved = bytes_spmv / (res["spmv_ms"] * 1e-3) / 1e9
    lu_bytes = res["lu_factor_bytes"]
    achieved_lu = lu_bytes / (res["lu_apply_ms"] * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_head,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-krylov/f64" if head == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME,
                   "precision": head, "newton_max": 5,
                   "krylov": "GMRES(30), multifrontal LU preconditioner (mixed: "
                             + ("FP32 factors" if args.lu_factors == "fp32"
                                else "FP64 factors rounded to FP32") + ")",
                   "lu_reuse_its": args.lu_reuse, "lu_reuse_steps": args.lu_reuse_steps,
                   "lu_solve": {"flow": "one dataflow launch", "levels": "one launch per level and sweep"}[args.lu_solve],
                   "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": world * res["e2e"]["steps_per_s"], "unit": "steps/s",
                "h2d_bytes_per_step": res["e2e"]["h2d"], "d2h_bytes_per_step": res["e2e"]["d2h"]},
        "roofline": {"bound": "hbm", "kernel": f"lu_apply_{prec_key} (the preconditioner "
                     "solve: k_solve_flow, or k_solve_level per level and sweep)",
                     "achieved": achieved_lu, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved_lu / peaks["hbm_gbs"], "traffic": None,
                     "traffic_note": "not measured in this run: ncu DRAM bytes of the same "
                                     "launch are in profiles/",
                     "bytes_per_launch": lu_bytes, "ms_per_launch": res["lu_apply_ms"],
                     "peak_note": peak_src},
        "roofline_spmv": {"bound": "hbm", "kernel": f"spmv_csr_{prec_key}",
                          "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                          "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                          "bytes_per_launch": bytes_spmv, "ms_per_launch": res["spmv_ms"]},
        "cpu_baseline": cpu,
        "kernel_rooflines": (kernel_rooflines(args.kernels_grid, peaks["hbm_gbs"])
                             if args.kernels_grid > 0 else None),
        "gpu_launches": int(launches.get(head, 0)),
        "clocks": res.get("clocks"),
        "legs": {p: res[p] for p in ("mixed", "fp64") if p in res},
        "lu_tuning": res.get("lu_tuning"),
    }
    if "mixed" in res and "fp64" in res:
        line["mixed_vs_fp64_speedup"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
        line["dCd_mixed_vs_fp64"] = abs(res["mixed"]["cd"] - res["fp64"]["cd"])
    print(jline(line), flush=True)


if __name__ == "__main__":
    main()
