"""Checkpoints of the dual-time state.

The file is a NumPy ``.npz`` archive with the members the reference's
checkpoints carry (vorti2d/restart.py:29-47), so either code base resumes the
other's runs:

    psi, ome, omeold, omeoldold   float64 arrays of imax*jmax (pointer order)
    t, step, imax, jmax, re       0-d arrays

A checkpoint is written to a temporary file in the destination folder and
moved into place, so a run killed while writing leaves the previous
checkpoint intact.
"""
from __future__ import annotations

import os
import tempfile
from dataclasses import dataclass

import numpy as np

FIELDS = ("psi", "ome", "omeold", "omeoldold")
SCALARS = (("t", float), ("step", int), ("imax", int), ("jmax", int), ("re", float))


@dataclass
class RestartState:
    """The four state fields plus time, step counter, grid size and Reynolds
    number (the BDF2 scheme needs both vorticity history levels to resume
    exactly)."""

    psi: np.ndarray
    ome: np.ndarray
    omeold: np.ndarray
    omeoldold: np.ndarray
    t: float
    step: int
    imax: int
    jmax: int
    re: float

    def __post_init__(self):
        for name, cast in SCALARS:
            setattr(self, name, cast(getattr(self, name)))


def _npz_path(path: str) -> str:
    # np.savez appends the suffix when it is missing; keep that naming
    return path if path.endswith(".npz") else path + ".npz"


def save_restart(path: str, st: RestartState) -> str:
    """Write ``st`` to ``path`` (``.npz`` appended when missing); returns the
    path written."""
    path = _npz_path(os.fspath(path))
    members = {name: np.asarray(getattr(st, name), dtype=np.float64) for name in FIELDS}
    members.update({name: np.asarray(getattr(st, name)) for name, _ in SCALARS})
    folder = os.path.dirname(os.path.abspath(path))
    fd, tmp = tempfile.mkstemp(prefix=".restart-", suffix=".npz", dir=folder)
    try:
        with os.fdopen(fd, "wb") as fh:
            np.savez(fh, **members)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise
    return path


def load_restart(path: str, imax: int, jmax: int) -> RestartState:
    """Read a checkpoint for an imax x jmax grid.  Raises ValueError when the
    file was written for another grid or lacks a member."""
    with np.load(path) as z:
        missing = [k for k in FIELDS + tuple(n for n, _ in SCALARS) if k not in z.files]
        if missing:
            raise ValueError(f"restart file {path} lacks {', '.join(missing)}")
        shape = (int(z["imax"]), int(z["jmax"]))
        if shape != (int(imax), int(jmax)):
            raise ValueError(f"restart mesh {shape[0]}x{shape[1]} != current mesh "
                             f"{imax}x{jmax}")
        fields = {k: np.ascontiguousarray(z[k], dtype=np.float64).reshape(-1) for k in FIELDS}
        for k, a in fields.items():
            if a.size != shape[0] * shape[1]:
                raise ValueError(f"restart field {k} has {a.size} values, expected "
                                 f"{shape[0] * shape[1]}")
        return RestartState(**fields, t=z["t"], step=z["step"], imax=imax, jmax=jmax,
                            re=z["re"])
