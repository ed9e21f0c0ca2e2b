"""Text output of a run, in the reference's file layout (vorti2d/fields_io.py:13-50,
columns of vorti2d/forces.py:79), so the reference's post-processing reads it:

    <out>/xg.csv, yg.csv                     the grid, one row per i
    <out>/psi_data/psi_tNNNN.csv             psi, one value per line
    <out>/omega_data/omega_tNNNN.csv         omega, one value per line
    <out>/residual_data/residual_history_tNNNN.csv   "iteration,log10(res)"
    <out>/forces.csv                         header + one row per step

Array files use 19 significant digits (``%.18e``) and forces.csv ``%.10e``,
comma separated.  NNNN is the physical step index, zero padded to 4 digits.
"""
from __future__ import annotations

import os

import numpy as np

SUBDIRS = {"psi": "psi_data", "omega": "omega_data", "residual": "residual_data"}
FORCES_FILE = "forces.csv"


def _fmt_rows(table: np.ndarray) -> str:
    """Rows of a 2-D float table as '%.18e' values joined by commas."""
    t = np.asarray(table, dtype=np.float64)
    if t.ndim == 1:
        t = t[:, None]
    return "".join(",".join(f"{v:.18e}" for v in row) + "\n" for row in t.tolist())


def _put(path: str, table) -> None:
    with open(path, "w") as fh:
        fh.write(_fmt_rows(table))


def step_file(out_dir: str, kind: str, step: int) -> str:
    """Path of the per-step file of `kind` ('psi', 'omega' or 'residual')."""
    stem = "residual_history" if kind == "residual" else kind
    return os.path.join(out_dir, SUBDIRS[kind], f"{stem}_t{int(step):04d}.csv")


def ensure_dirs(out_dir: str):
    for sub in SUBDIRS.values():
        os.makedirs(os.path.join(out_dir, sub), exist_ok=True)


def write_fields(out_dir: str, step: int, psi: np.ndarray, ome: np.ndarray):
    _put(step_file(out_dir, "psi", step), np.ravel(psi))
    _put(step_file(out_dir, "omega", step), np.ravel(ome))


def write_residual_history(out_dir: str, step: int, res_log10):
    r = np.asarray(res_log10, dtype=np.float64).ravel()
    _put(step_file(out_dir, "residual", step),
         np.stack([np.arange(1, r.size + 1, dtype=np.float64), r], axis=1))


def write_grid(out_dir: str, xg: np.ndarray, yg: np.ndarray):
    _put(os.path.join(out_dir, "xg.csv"), np.atleast_2d(xg))
    _put(os.path.join(out_dir, "yg.csv"), np.atleast_2d(yg))


def init_force_history(out_dir: str, columns):
    """Start forces.csv with its header line; returns its path."""
    path = os.path.join(out_dir, FORCES_FILE)
    with open(path, "w") as fh:
        fh.write(",".join(columns) + "\n")
    return path


def append_force_history(out_dir: str, columns, row: dict):
    """Add one step's coefficients (``row`` keyed by ``columns``)."""
    line = ",".join(format(float(row[c]), ".10e") for c in columns)
    with open(os.path.join(out_dir, FORCES_FILE), "a") as fh:
        fh.write(line + "\n")
