"""In-house autotuner of the LU preconditioner solve's work-item granularity.

The solve (one dataflow launch over the front tree) runs in one of two
kernel forms (more resident CTAs per SM, or more row registers per lane) and
splits each front's rows
into work items; on tree level L an item is ``rows[L]`` rows of one front, or
the whole front (0), or, for ``rows[L] = -R``, R rows after one gather item
per front that collects the front's right-hand side once for all of its
items.  Small items spread a level's rows over more CTAs and shorten the
chain of dependent steps; large ones gather each front's right-hand side once
and keep a CTA's rows together; gather items add one dependent step but
spare every item the indexed gather.  Which wins depends on
the grid, the precision and the GPU, so it is measured: a coordinate search
over the levels (each level's candidates tried with the others fixed, two
sweeps), then the split form (the lower levels as launches of their own with
smaller CTAs, ``split`` levels, followed by one more sweep over those
levels' rows), every trial timed as the average of warm applications of the
current factors (``v2d_solver_time_lu_apply``, factors in L2 as inside
GMRES).  Every setting forms the same products; a row's partial sums are
added in an order that depends on the split, so results agree to rounding
and each Krylov solve still meets its tolerance.

The result can be written to a JSON file keyed by grid shape, precision and
leaf size, and read back (``Config.lu_item_rows``, ``load_tuning``).
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from . import _lib
from ._lib import check, lib

# rows per item: 0 whole fronts, R > 0 R-row items, R < 0 (-R)-row items
# after one gather item per split front
CANDIDATES = (0, 8, 16, 32, 64, 128, 256, -8, -16, -32, -64, -128, -256)


def item_rows(solver) -> list:
    """The solve's current rows per item, one entry per tree level."""
    n = ctypes.c_int()
    check(lib().v2d_solver_lu_item_rows(solver.dev.h, None, 0, None, 0, ctypes.byref(n)),
          "lu_item_rows")
    out = np.zeros(n.value, dtype=np.intc)
    check(lib().v2d_solver_lu_item_rows(solver.dev.h, None, 0, _lib.iptr(out), n.value, None),
          "lu_item_rows")
    return [int(v) for v in out]


def set_item_rows(solver, rows) -> None:
    r = np.ascontiguousarray(rows, dtype=np.intc)
    check(lib().v2d_solver_lu_item_rows(solver.dev.h, _lib.iptr(r), r.size, None, 0, None),
          "lu_item_rows")


def flow_form(solver) -> int:
    cur = ctypes.c_int()
    check(lib().v2d_solver_lu_flow_form(solver.dev.h, -1, ctypes.byref(cur)), "lu_flow_form")
    return cur.value


def set_flow_form(solver, form: int) -> bool:
    """Select a form of the dataflow solve kernel; False when the solve has
    no such form on this GPU."""
    return lib().v2d_solver_lu_flow_form(solver.dev.h, int(form), None) == _lib.V2D_OK


def split_level(solver) -> int:
    cur = ctypes.c_int()
    check(lib().v2d_solver_lu_split(solver.dev.h, -1, ctypes.byref(cur)), "lu_split")
    return cur.value


def set_split_level(solver, level: int) -> bool:
    """Run the tree levels [0, level) of the solve as launches of their own
    (0: one launch); False when the setting does not fit."""
    return lib().v2d_solver_lu_split(solver.dev.h, int(level), None) == _lib.V2D_OK


def time_apply(solver, reps: int = 30, repeats: int = 3) -> float:
    """ms of one warm LU application: the smallest of `repeats` averages of
    `reps` applications."""
    best = float("inf")
    for _ in range(repeats):
        ms, fb = ctypes.c_double(), ctypes.c_longlong()
        check(lib().v2d_solver_time_lu_apply(solver.dev.h, int(reps), 0, ctypes.byref(ms),
                                             ctypes.byref(fb)), "time_lu_apply")
        best = min(best, ms.value)
    return best


def _key(solver) -> str:
    cfg = solver.cfg
    return f"{solver.imax}x{solver.jmax}/{cfg.precision}/{cfg.lu_factors}"


def tune_lu_solve(solver, candidates=CANDIDATES, sweeps: int = 2, reps: int | None = None,
                  path: str | None = None, gain: float = 0.01) -> dict:
    """Tune the solver's rows per item in place (its factors must exist: run a
    Newton iteration first).  A trial replaces the current choice when it is
    faster by more than `gain` (relative).  `reps` applications per timing
    (default: about 10 ms of them, 3 to 30).  Returns the record (and merges
    it into the JSON file at `path` when given)."""
    rows = item_rows(solver)
    if reps is None:
        reps = int(min(30, max(3, round(10.0 / max(time_apply(solver, 3, 1), 1e-3)))))
    t0 = time_apply(solver, reps)
    best = t0
    trials = 0
    # kernel form first (resident CTAs per SM against row registers)
    form = flow_form(solver)
    for f in (0, 1):
        if f == form or not set_flow_form(solver, f):
            continue
        t = time_apply(solver, reps)
        trials += 1
        if t < best * (1.0 - gain):
            best, form = t, f
    set_flow_form(solver, form)
    def sweep(levels):
        nonlocal best, rows, trials
        changed = False
        for L in levels:
            for c in candidates:
                if c == rows[L]:
                    continue
                trial = list(rows)
                trial[L] = int(c)
                set_item_rows(solver, trial)
                t = time_apply(solver, reps)
                trials += 1
                if t < best * (1.0 - gain):
                    best, rows, changed = t, trial, True
            set_item_rows(solver, rows)
        return changed

    for _ in range(sweeps):
        if not sweep(range(len(rows))):
            break
    set_item_rows(solver, rows)
    # split form: the lower levels as launches of their own, then their rows
    # again under it
    split = split_level(solver)
    for lv in range(1, min(len(rows), 9)):
        if lv == split or not set_split_level(solver, lv):
            continue
        t = time_apply(solver, reps)
        trials += 1
        if t < best * (1.0 - gain):
            best, split = t, lv
    set_split_level(solver, split)
    if split > 0:
        sweep(range(split))
    set_item_rows(solver, rows)
    rec = {"key": _key(solver), "rows": rows, "form": form, "split": split, "ms": best,
           "default_ms": t0, "trials": trials, "reps": reps, "candidates": list(candidates)}
    if path:
        table = {}
        if os.path.exists(path):
            with open(path) as fh:
                table = json.load(fh)
        table[rec["key"]] = rec
        tmp = path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(table, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    return rec


def load_tuning(solver, path: str) -> bool:
    """Apply the rows recorded for this solver's grid and precision in the
    JSON file at `path`; False when the file has none (the default split
    stays)."""
    if not os.path.exists(path):
        return False
    with open(path) as fh:
        rec = json.load(fh).get(_key(solver))
    if not rec or len(rec.get("rows", [])) != len(item_rows(solver)):
        return False
    set_item_rows(solver, rec["rows"])
    set_flow_form(solver, rec.get("form", 0))
    set_split_level(solver, rec.get("split", 0))
    return True
