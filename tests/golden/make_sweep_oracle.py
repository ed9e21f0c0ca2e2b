"""The oracle's steady solves of the 96-instance sweep (CPU, one process per
core, a few minutes):

    python tests/golden/make_sweep_oracle.py [--procs 8] [--out FILE]

Cases: vorti2d_b200.batch.sweep_cases(seed 0) -- 32 cylinders 129x129, 32
cylinders 181x181, 32 NACA-0012 sections 257x129, Re ~ U[50, 1000], alpha ~
U[-8, 8] degrees.  Each case runs the reference's steady loop
(vorti2d/solver.py:136-145, pure Newton from the free stream, SuperLU standing
in for MUMPS) with the batched sweep's stopping rules: at most 20 Newton
iterations, converged when ||dq||/(2N) <= 1e-10, diverged when ||dq||/(2N)
exceeds 1000 times its first value or is not finite.

Stored (JSON): per case its name, Re, alpha, whether it converged, the
Newton iterations, the update norms, and Cd / Cl / Cm of converged cases.
The GPU test tests/test_gpu_batch_forest.py runs the same sweep batched on
the device and compares the converged set and the forces.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MAX_NEWTON = 20
TOL = 1e-10
DIVERGE = 1e3


def solve_case(args):
    name, xg, yg, re, alpha, ref_length = args
    import numpy as np
    from oracle import oracle as O
    s = O.OracleSolver(xg, yg, re=re, steady=True, alpha_deg=alpha, pseudo_tol=TOL,
                       max_pseudo_iter=MAX_NEWTON, ref_length=ref_length)
    res_log = []
    status = "max_iter"
    for _ in range(MAX_NEWTON):
        try:
            res = s.newton_once(0.0)
        except Exception as exc:   # a singular or non-finite system counts as diverged
            status = f"error: {type(exc).__name__}"
            break
        res_log.append(res)
        if not math.isfinite(res) or res > DIVERGE * res_log[0]:
            status = "diverged"
            break
        if res <= TOL:
            status = "converged"
            break
    out = {"name": name, "re": re, "alpha_deg": alpha, "status": status,
           "converged": status == "converged", "newton_its": len(res_log),
           "res": [float(r) for r in res_log]}
    if out["converged"]:
        fc = O.compute_force_coeffs(s.imax, s.jmax, re, s.dksi, s.deta, s.beta, s.gama,
                                    s.detadx, s.detady, s.xphys, s.yphys, s.ome,
                                    ref_length=ref_length)
        out.update(cd=float(fc.cd), cl=float(fc.cl), cm=float(fc.cm))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=os.path.join(HERE, "sweep_oracle_96.json"))
    a = ap.parse_args()
    from vorti2d_b200.batch import sweep_cases
    cases = sweep_cases(seed=0)
    work = [(c.name, c.xg, c.yg, c.re, c.alpha_deg, c.ref_length) for c in cases]
    t0 = time.time()
    with mp.get_context("spawn").Pool(a.procs) as pool:
        rows = pool.map(solve_case, work, chunksize=1)
    rec = {"seed": 0, "max_newton": MAX_NEWTON, "tol": TOL, "diverge_factor": DIVERGE,
           "solver": "oracle: C restatement of vorti2d_core.f90 + SuperLU, pure Newton",
           "seconds": time.time() - t0, "cases": rows}
    with open(a.out, "w") as fh:
        json.dump(rec, fh, indent=1)
    conv = [r["name"] for r in rows if r["converged"]]
    print(f"{len(conv)} of {len(rows)} converged in {rec['seconds']:.0f} s: {conv}")


if __name__ == "__main__":
    main()
