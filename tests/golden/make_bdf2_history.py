"""Generate the long-horizon fixture of the unsteady cylinder benchmark from
the oracle (CPU, single process, about 30 minutes):

    python tests/golden/make_bdf2_history.py [--steps 400] [--out FILE]

Workload: cylinder O-grid 181x181 from the reference's generator
(vorti2d/mesh.py:14-50, inner radius 0.5, outer 50), Re=100, BDF2 with
dt=0.2, rotational kick 0.5 until t=2, outflow far field, at most 5 Newton
iterations per step to ||dq||/(2N) <= 1e-10 -- the reference's replicated
driver (vorti2d/solver.py:169-217) with SuperLU standing in for MUMPS.

Stored (np.savez_compressed):
  t, cd, cl, cm         per step, after the step's Newton iterations
  newton_its, newton_res per step
  ckpt_steps            step indices whose fields are stored
  psi_ckpt, ome_ckpt    (len(ckpt_steps), N) fields after those steps
  st, st_window         Strouhal number of the lift over the trailing
                        window (zero crossings, see strouhal())
The GPU test tests/test_gpu_bdf2_history.py replays the same steps on the
device and compares against this file.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

WORKLOAD = dict(re=100.0, steady=False, dt_phys=0.2, rot_speed=0.5, rot_until=2.0,
                farfield_bc="outflow")
NEWTON = dict(pseudo_tol=1e-10, max_pseudo_iter=5)
GRID = (181, 181)
CKPT = (24, 100, 399)


def strouhal(t, cl, t_from):
    """Lift frequency from the upward zero crossings of cl - mean(cl) with
    t >= t_from, linearly interpolated between samples (D = U = 1, so St = f).
    Returns (St, number of full periods used); (nan, 0) without two crossings."""
    t = np.asarray(t, dtype=np.float64)
    cl = np.asarray(cl, dtype=np.float64)
    m = t >= t_from
    tt, cc = t[m], cl[m] - np.mean(cl[m])
    ups = [tt[k] - cc[k] * (tt[k + 1] - tt[k]) / (cc[k + 1] - cc[k])
           for k in range(len(tt) - 1) if cc[k] < 0.0 <= cc[k + 1]]
    if len(ups) < 2:
        return float("nan"), 0
    return float((len(ups) - 1) / (ups[-1] - ups[0])), len(ups) - 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--out", default=os.path.join(HERE, "bdf2_history_181.npz"))
    args = ap.parse_args()
    from oracle import oracle as O
    xg, yg = O.generate_cylinder(*GRID)
    t_end = 0.2 * (args.steps - 1)
    s = O.OracleSolver(xg, yg, t_end=t_end, **NEWTON, **WORKLOAD)
    times = s.times()[:args.steps]
    ckpt = [c for c in CKPT if c < args.steps]
    rec = {k: [] for k in ("t", "cd", "cl", "cm", "newton_its", "newton_res")}
    psi_ck, ome_ck = [], []
    t0 = time.time()
    for m, t in enumerate(times):
        res, it = s.advance(t)
        fc = s.force_coeffs()
        for k, v in (("t", t), ("cd", fc.cd), ("cl", fc.cl), ("cm", fc.cm),
                     ("newton_its", it), ("newton_res", res)):
            rec[k].append(v)
        if m in ckpt:
            psi_ck.append(s.psi.copy())
            ome_ck.append(s.ome.copy())
        print(f"step {m} t={t:.1f} its={it} res={res:.3e} cd={fc.cd:.10f} cl={fc.cl:+.10f} "
              f"({time.time() - t0:.0f} s)", flush=True)
    t_from = 0.5 * times[-1]
    st, periods = strouhal(rec["t"], rec["cl"], t_from)
    print(f"St = {st:.5f} over {periods} periods from t = {t_from:.1f}")
    np.savez_compressed(
        args.out, imax=GRID[0], jmax=GRID[1], **{k: np.asarray(v) for k, v in rec.items()},
        ckpt_steps=np.asarray(ckpt, dtype=np.int64), psi_ckpt=np.asarray(psi_ck),
        ome_ckpt=np.asarray(ome_ck), st=st, st_window=t_from)


if __name__ == "__main__":
    main()
