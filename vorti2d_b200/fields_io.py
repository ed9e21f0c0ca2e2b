"""Field / history output, format-compatible with vorti2d/fields_io.py:13-50
(MATLAB-style psi/omega column CSVs, residual history, forces.csv)."""
from __future__ import annotations

import os

import numpy as np


def ensure_dirs(out_dir: str):
    for sub in ("psi_data", "omega_data", "residual_data"):
        os.makedirs(os.path.join(out_dir, sub), exist_ok=True)


def write_fields(out_dir: str, step: int, psi: np.ndarray, ome: np.ndarray):
    np.savetxt(os.path.join(out_dir, "psi_data", f"psi_t{step:04d}.csv"),
               psi.reshape(-1, 1), delimiter=",")
    np.savetxt(os.path.join(out_dir, "omega_data", f"omega_t{step:04d}.csv"),
               ome.reshape(-1, 1), delimiter=",")


def write_residual_history(out_dir: str, step: int, res_log10):
    n = len(res_log10)
    table = np.column_stack((np.arange(1, n + 1), np.asarray(res_log10, dtype=np.float64)))
    np.savetxt(os.path.join(out_dir, "residual_data", f"residual_history_t{step:04d}.csv"),
               table, delimiter=",")


def write_grid(out_dir: str, xg: np.ndarray, yg: np.ndarray):
    np.savetxt(os.path.join(out_dir, "xg.csv"), xg, delimiter=",")
    np.savetxt(os.path.join(out_dir, "yg.csv"), yg, delimiter=",")


def init_force_history(out_dir: str, columns):
    path = os.path.join(out_dir, "forces.csv")
    with open(path, "w") as fh:
        fh.write(",".join(columns) + "\n")
    return path


def append_force_history(out_dir: str, columns, row: dict):
    path = os.path.join(out_dir, "forces.csv")
    with open(path, "a") as fh:
        fh.write(",".join(f"{row[c]:.10e}" for c in columns) + "\n")
