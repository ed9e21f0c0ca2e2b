"""Mesh handling (drop-in for ``vorti2d.mesh``, vorti2d/mesh.py).

Meshes are (imax, jmax) arrays: i circumferential with the branch cut at
i=0 == i=imax-1, j radial with j=0 the wall and j=jmax-1 the far field.
"""
from __future__ import annotations

import numpy as np


def generate_cylinder(imax: int = 181, jmax: int = 181, inner_rad: float = 0.5,
                      outer_rad: float = 50.0):
    """Cylinder O-grid with the reference's algebraic clustering
    (vorti2d/mesh.py:14-50): radial increments 1, 1, 1, 2, 3, ... normalised,
    circumferential weights min(i, imax-i)**0.6, theta = 2 pi (1 - s_i)."""
    alen = np.zeros(jmax)
    for jm in range(1, min(jmax, 4)):
        alen[jm] = float(jm)
    for jm in range(4, jmax):
        alen[jm] = alen[jm - 1] + (jm - 2)
    alen /= alen[jmax - 1]
    alen2 = np.zeros(imax)
    for im in range(1, imax):
        alen2[im] = alen2[im - 1] + min(im, imax - im) ** 0.6
    alen2 /= alen2[imax - 1]
    theta = 2.0 * np.pi * (1.0 - alen2)
    rad = inner_rad + (outer_rad - inner_rad) * alen
    xg = rad[None, :] * np.cos(theta)[:, None]
    yg = rad[None, :] * np.sin(theta)[:, None]
    return xg, yg


def save_mesh(xg: np.ndarray, yg: np.ndarray, xg_path: str, yg_path: str):
    """Write a mesh to two CSV files (vorti2d/mesh.py:53-56)."""
    np.savetxt(xg_path, xg, delimiter=",")
    np.savetxt(yg_path, yg, delimiter=",")


def load_mesh(xg_path: str, yg_path: str):
    """Read a mesh from two CSV files (vorti2d/mesh.py:59-68)."""
    xg = np.loadtxt(xg_path, delimiter=",")
    yg = np.loadtxt(yg_path, delimiter=",")
    if xg.shape != yg.shape:
        raise ValueError(f"xg shape {xg.shape} != yg shape {yg.shape}")
    if xg.ndim != 2:
        raise ValueError("mesh CSVs must be 2-D (imax x jmax)")
    return np.ascontiguousarray(xg, dtype=np.float64), np.ascontiguousarray(yg, dtype=np.float64)


def load_cgns_ogrid(cgns_path: str, plane: int = 0, block: int = 0, verbose: bool = False):
    """pyHyp CGNS reader (vorti2d/mesh.py:93-140).  Needs ``cgnsutilities``,
    which vorti2d_b200 does not depend on; convert the grid to xg/yg CSV instead."""
    try:
        import cgnsutilities  # noqa: F401
    except ImportError as exc:
        raise NotImplementedError(
            "load_cgns_ogrid needs cgnsutilities, which is not installed; "
            "export the O-grid to xg/yg CSV and use load_mesh") from exc
    raise NotImplementedError("CGNS import is outside the GPU hot path")


def naca00xx_thickness(x: np.ndarray, t: float = 0.12) -> np.ndarray:
    """Half-thickness of the NACA 4-digit symmetric section (open trailing
    edge form, coefficients 0.2969, -0.1260, -0.3516, 0.2843, -0.1015)."""
    return 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3
                      - 0.1015 * x ** 4)


def generate_naca0012(imax: int = 257, jmax: int = 129, chord: float = 1.0,
                      farfield: float = 30.0, thickness: float = 0.12,
                      first_cell: float | None = None):
    """NACA-0012 O-grid from the analytic thickness formula with algebraic
    normal extrusion to ``farfield`` chords.

    The section is centred at mid-chord (no wall node at the origin, where the
    rotating-wall vorticity condition would divide by zero).  The open
    trailing edge is closed by a short base whose midpoint carries the branch
    cut (i = 0 == imax-1).  Surface nodes follow the cylinder generator's
    orientation (clockwise: the lower surface first).  Each grid line leaves
    the wall along the surface normal and blends into a circle of radius
    ``farfield * chord`` around mid-chord; radial spacing grows geometrically
    from ``first_cell`` (default chord/(4 (jmax-1)))."""
    if imax < 9 or jmax < 4:
        raise ValueError("NACA O-grid needs imax >= 9 and jmax >= 4")
    P = imax - 1                                   # distinct surface nodes
    # surface parameter s in [0, 1): 0 = trailing-edge base midpoint (seam)
    s = np.arange(P) / P
    # arc parameter around the closed section: lower TE -> LE -> upper TE
    ang = 2.0 * np.pi * s                          # 0 .. 2 pi
    xc = 0.5 * (1.0 + np.cos(ang))                 # 1 at TE, 0 at LE (cosine clustering)
    yt = naca00xx_thickness(xc, thickness)
    lower = ang < np.pi
    ys = np.where(lower, -yt, yt)
    xs = (xc - 0.5) * chord
    ys = ys * chord
    # the seam node sits on the base midpoint (x = TE, y = 0)
    xs[0], ys[0] = 0.5 * chord, 0.0
    # outward normals from the periodic central tangent
    tx = np.roll(xs, -1) - np.roll(xs, 1)
    ty = np.roll(ys, -1) - np.roll(ys, 1)
    tn = np.hypot(tx, ty)
    nx, ny = ty / tn, -tx / tn                     # clockwise traversal: outward = (ty, -tx)
    # make sure normals point away from the centre
    if np.mean(nx * xs + ny * ys) < 0:
        nx, ny = -nx, -ny
    # radial distribution: geometric growth to the far field
    R = farfield * chord
    h0 = first_cell if first_cell is not None else chord / (4.0 * (jmax - 1))
    ncell = jmax - 1
    # solve h0 (q^ncell - 1)/(q - 1) = R for q
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if h0 * (mid ** ncell - 1.0) / (mid - 1.0) > R:
            hi = mid
        else:
            lo = mid
    q = 0.5 * (lo + hi)
    dist = np.concatenate([[0.0], h0 * (q ** np.arange(1, ncell + 1) - 1.0) / (q - 1.0)])
    dist *= R / dist[-1]
    w = dist / R                                   # 0 at the wall, 1 at the far field
    blend = w ** 2 * (3.0 - 2.0 * w)               # smooth transition to the circle
    # far-field circle at uniform angles in the surface parameter (clockwise,
    # like the surface): arctan2 of the surface points would crowd the lines
    # next to the thin trailing edge onto nearly one angle and fold the outer
    # cells beside the seam
    phi = -ang
    xo, yo = R * np.cos(phi), R * np.sin(phi)
    xg = np.empty((imax, jmax))
    yg = np.empty((imax, jmax))
    xn = xs[:, None] + dist[None, :] * nx[:, None]
    yn = ys[:, None] + dist[None, :] * ny[:, None]
    xg[:P] = (1.0 - blend[None, :]) * xn + blend[None, :] * xo[:, None]
    yg[:P] = (1.0 - blend[None, :]) * yn + blend[None, :] * yo[:, None]
    xg[P] = xg[0]
    yg[P] = yg[0]
    return xg, yg
