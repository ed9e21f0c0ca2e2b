"""Drop-in for the f2py module ``vorti2d.core`` (= ``vorti2d._core.vorti2d_core``).

Same five routines, same argument order and return tuples as the reference's
f2py wrapper of src/fortran/vorti2d_core.f90 (hidden dimensions inferred from
the arrays, outputs freshly allocated), computed by the sm_100a kernels of
libvorti2d_b200.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, dptr, f64, iptr, lib


def _fortran2d(a, name):
    a = np.asarray(a, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError(f"{name} must be a 2-D array (imax, jmax)")
    return np.asfortranarray(a)


class _Core:
    """Namespace object mirroring ``vorti2d._core.vorti2d_core``."""

    # vorti2d_core.f90:33-61
    @staticmethod
    def node_neighbors(i, j, imax):
        out = np.zeros(9, dtype=np.intc)
        check(lib().v2d_node_neighbors(int(i), int(j), int(imax), iptr(out)), "node_neighbors")
        return tuple(int(v) for v in out)

    # vorti2d_core.f90:66-189 (vorti2d/solver.py:72-74)
    @staticmethod
    def compute_metrics(dksi, deta, xg, yg):
        xg = _fortran2d(xg, "xg")
        yg = _fortran2d(yg, "yg")
        if xg.shape != yg.shape:
            raise ValueError(f"xg shape {xg.shape} != yg shape {yg.shape}")
        imax, jmax = xg.shape
        outs = [np.zeros(imax * jmax) for _ in range(10)]
        check(lib().v2d_compute_metrics(imax, jmax, float(dksi), float(deta), dptr(xg), dptr(yg),
                                        *[dptr(o) for o in outs]), "compute_metrics")
        return tuple(outs)

    # vorti2d_core.f90:392-495 (vorti2d/dist_solver.py:92-93)
    @staticmethod
    def compute_metrics_local(il0, il1, dksi, deta, xgl, ygl):
        xgl = _fortran2d(xgl, "xgl")
        ygl = _fortran2d(ygl, "ygl")
        if xgl.shape != ygl.shape:
            raise ValueError(f"xgl shape {xgl.shape} != ygl shape {ygl.shape}")
        gxm, jmax = xgl.shape
        outs = [np.zeros(gxm * jmax) for _ in range(10)]
        check(lib().v2d_compute_metrics_local(gxm, jmax, int(il0), int(il1), float(dksi),
                                              float(deta), dptr(xgl), dptr(ygl),
                                              *[dptr(o) for o in outs]), "compute_metrics_local")
        return tuple(outs)

    # vorti2d_core.f90:219-383 (vorti2d/solver.py:121-127)
    @staticmethod
    def assemble_coo(imax, jmax, re, invdtau, inv2dt, urot, dksi, deta, jac, alfa, beta, gama,
                     pmet, qmet, detadx, detady, xphys, yphys, psi, ome, omeold, omeoldold,
                     r0, r1, maxnnz, ff_bc, ca, sa):
        N = int(imax) * int(jmax)
        arrs = [f64(a) for a in (jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys,
                                 yphys, psi, ome, omeold, omeoldold)]
        for a in arrs:
            if a.size != N:
                raise ValueError(f"field arrays must have imax*jmax = {N} entries (got {a.size})")
        ci = np.zeros(int(maxnnz), dtype=np.intc)
        cj = np.zeros(int(maxnnz), dtype=np.intc)
        cv = np.zeros(int(maxnnz))
        bvec = np.zeros(int(r1) - int(r0))
        nnz = ctypes.c_int(0)
        check(lib().v2d_assemble_coo(int(imax), int(jmax), float(re), float(invdtau),
                                     float(inv2dt), float(urot), float(dksi), float(deta),
                                     *[dptr(a) for a in arrs], int(r0), int(r1), int(maxnnz),
                                     int(ff_bc), float(ca), float(sa), iptr(ci), iptr(cj),
                                     dptr(cv), ctypes.byref(nnz), dptr(bvec)), "assemble_coo")
        return ci, cj, cv, nnz.value, bvec

    # vorti2d_core.f90:510-661 (vorti2d/dist_solver.py:310-317)
    @staticmethod
    def assemble_coo_local(gxm, jmax, il0, il1, re, invdtau, inv2dt, urot, dksi, deta, jac,
                           alfa, beta, gama, pmet, qmet, detadx, detady, xphys, yphys, psi, ome,
                           omeold, omeoldold, r0, nloc, lg, maxnnz, ff_bc, ca, sa):
        N = int(gxm) * int(jmax)
        arrs = [f64(a) for a in (jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys,
                                 yphys, psi, ome, omeold, omeoldold)]
        for a in arrs:
            if a.size != N:
                raise ValueError(f"local arrays must have gxm*jmax = {N} entries (got {a.size})")
        lg = np.ascontiguousarray(lg, dtype=np.intc)
        if lg.size != 2 * N:
            raise ValueError(f"lg must have 2*gxm*jmax = {2 * N} entries (got {lg.size})")
        ci = np.zeros(int(maxnnz), dtype=np.intc)
        cj = np.zeros(int(maxnnz), dtype=np.intc)
        cv = np.zeros(int(maxnnz))
        bvec = np.zeros(int(nloc))
        nnz = ctypes.c_int(0)
        check(lib().v2d_assemble_coo_local(int(gxm), int(jmax), int(il0), int(il1), float(re),
                                           float(invdtau), float(inv2dt), float(urot),
                                           float(dksi), float(deta), *[dptr(a) for a in arrs],
                                           int(r0), int(nloc), iptr(lg), int(maxnnz), int(ff_bc),
                                           float(ca), float(sa), iptr(ci), iptr(cj), dptr(cv),
                                           ctypes.byref(nnz), dptr(bvec)), "assemble_coo_local")
        return ci, cj, cv, nnz.value, bvec


vorti2d_core = _Core()
