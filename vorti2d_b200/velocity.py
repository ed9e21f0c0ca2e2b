"""Velocity reconstruction (drop-in for ``vorti2d.velocity``,
vorti2d/velocity.py:38-93): u = dpsi/dy, v = -dpsi/dx on the curvilinear
O-grid, evaluated on the GPU by ``v2d_compute_velocity``."""
from __future__ import annotations

import numpy as np

from ._lib import check, dptr, f64, lib


def xi_gradients(jac, beta, gama, detadx, detady):
    """(xi_x, xi_y) from the exported metrics (vorti2d/velocity.py:38-43):
    xi_x = (gamma eta_x + J eta_y) / beta, xi_y = (gamma eta_y - J eta_x) / beta.
    A host helper for post-processing; the device kernel recomputes these
    per node."""
    jac, beta, gama, detadx, detady = (f64(a) for a in (jac, beta, gama, detadx, detady))
    return (gama * detadx + jac * detady) / beta, (gama * detady - jac * detadx) / beta


def compute_velocity(imax: int, jmax: int, dksi: float, deta: float, jac, beta, gama, detadx,
                     detady, psi, want_mag: bool = False):
    """Cartesian velocity ``(u, v[, |V|])`` from a psi field
    (vorti2d/velocity.py:76-93); arrays of imax*jmax in pointer order."""
    arrs = [f64(a) for a in (jac, beta, gama, detadx, detady, psi)]
    N = int(imax) * int(jmax)
    for a in arrs:
        if a.size != N:
            raise ValueError(f"arrays must have imax*jmax = {N} entries (got {a.size})")
    u, v = np.empty(N), np.empty(N)
    mag = np.empty(N) if want_mag else None
    check(lib().v2d_compute_velocity(int(imax), int(jmax), float(dksi), float(deta),
                                     *[dptr(a) for a in arrs], dptr(u), dptr(v),
                                     dptr(mag) if want_mag else None), "compute_velocity")
    return (u, v, mag) if want_mag else (u, v)
