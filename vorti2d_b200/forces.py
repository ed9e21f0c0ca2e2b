"""Force / moment coefficients (drop-in for ``vorti2d.forces``).

``compute_force_coeffs`` keeps the reference signature
(vorti2d/forces.py:82-194) and evaluates the wall integrals on the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass, asdict

import numpy as np

from ._lib import check, dptr, f64, lib


@dataclass
class ForceCoeffs:
    """Force / moment coefficients and their pressure / friction split
    (vorti2d/forces.py:60-75)."""
    cd: float
    cl: float
    cm: float
    cdp: float
    cdf: float
    clp: float
    clf: float
    cmp: float
    cmf: float
    ref_length: float

    def to_dict(self) -> dict:
        return asdict(self)

    @classmethod
    def from_array(cls, out) -> "ForceCoeffs":
        return cls(*[float(v) for v in out])


FORCE_COLUMNS = ("t", "cd", "cl", "cm", "cdp", "cdf", "clp", "clf", "cmp", "cmf")


def compute_force_coeffs(imax: int, jmax: int, re: float, dksi: float, deta: float,
                         beta: np.ndarray, gama: np.ndarray, detadx: np.ndarray,
                         detady: np.ndarray, xphys: np.ndarray, yphys: np.ndarray,
                         ome: np.ndarray, ref_length: float | None = None,
                         moment_ref: tuple[float, float] = (0.0, 0.0)) -> ForceCoeffs:
    arrs = [f64(a) for a in (beta, gama, detadx, detady, xphys, yphys, ome)]
    N = int(imax) * int(jmax)
    for a in arrs:
        if a.size != N:
            raise ValueError(f"arrays must have imax*jmax = {N} entries (got {a.size})")
    out = np.zeros(10)
    rl = -1.0 if ref_length is None else float(ref_length)
    check(lib().v2d_force_coeffs(int(imax), int(jmax), float(re), float(dksi), float(deta),
                                 *[dptr(a) for a in arrs], rl, float(moment_ref[0]),
                                 float(moment_ref[1]), dptr(out)), "compute_force_coeffs")
    return ForceCoeffs.from_array(out)
