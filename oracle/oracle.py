"""ORACLE -- test infrastructure only.

CPU restatement of the vorti2d hot path, used by ``tests/``, by
``__graft_entry__.smoke()`` as the checker, and by ``bench.py``'s
``cpu_baseline`` / ``--impl reference`` legs as the timed CPU baseline.  The
product package (``vorti2d_b200``) never imports this module.

Pieces (each cites the reference file:line it restates):

* ``OracleCore`` -- ctypes binding of ``oracle/v2d_oracle.c`` (a line-by-line C
  restatement of ``src/fortran/vorti2d_core.f90``) with the f2py call
  signatures of ``vorti2d.core`` (outputs freshly allocated, hidden dims
  inferred from the arrays).
* ``generate_cylinder`` -- ``vorti2d/mesh.py:14-50``.
* ``compute_force_coeffs`` -- ``vorti2d/forces.py:82-194``.
* ``OracleSolver`` -- ``vorti2d/solver.py:48-224`` with the linear solve of
  ``vorti2d/petsc_solver.py:76-115`` (scipy canonical CSR; scipy SuperLU
  ``spsolve`` stands in for MUMPS, both direct LU).

Parity anchor: the reference's Fortran and PETSc layers cannot be built in this
image; the restatement is pinned by the reference's known-answer tests and
documented drag values (see ``tests/test_oracle_known_answers.py``) and, for
the pure-NumPy modules, by golden vectors generated from the reference's own
``mesh.py`` / ``forces.py`` (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, asdict

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "v2d_oracle.c")
_LIB = os.path.join(_HERE, "_build", "libv2d_oracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc, no fast-math, no FP contraction)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        os.makedirs(os.path.dirname(_LIB), exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-fno-fast-math", "-ffp-contract=off",
                               "-fPIC", "-shared", "-o", _LIB, _SRC, "-lm"])
    return _LIB


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleCore:
    """f2py-shaped wrapper around the C restatement (``vorti2d.core`` surface)."""

    def __init__(self):
        self.lib = ctypes.CDLL(build())
        L = self.lib
        L.v2d_oracle_node_neighbors.argtypes = [ctypes.c_int] * 3 + [_ip]
        L.v2d_oracle_compute_metrics.argtypes = ([ctypes.c_int] * 2 + [ctypes.c_double] * 2
                                                 + [_dp] * 12)
        L.v2d_oracle_compute_metrics_local.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_double] * 2
                                                       + [_dp] * 12)
        L.v2d_oracle_assemble_coo.argtypes = ([ctypes.c_int] * 2 + [ctypes.c_double] * 6
                                              + [_dp] * 14 + [ctypes.c_int] * 4
                                              + [ctypes.c_double] * 2 + [_ip, _ip, _dp, _ip, _dp])
        L.v2d_oracle_assemble_coo_local.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_double] * 6
                                                    + [_dp] * 14 + [ctypes.c_int] * 2 + [_ip]
                                                    + [ctypes.c_int] * 2
                                                    + [ctypes.c_double] * 2
                                                    + [_ip, _ip, _dp, _ip, _dp])

    # vorti2d_core.f90:33-61
    def node_neighbors(self, i, j, imax):
        out = np.zeros(9, dtype=np.intc)
        self.lib.v2d_oracle_node_neighbors(int(i), int(j), int(imax), _ptr(out, _ip))
        return tuple(int(v) for v in out)

    # vorti2d_core.f90:66-189 ; f2py: compute_metrics(dksi, deta, xg, yg)
    def compute_metrics(self, dksi, deta, xg, yg):
        xg = np.asfortranarray(xg, dtype=np.float64)
        yg = np.asfortranarray(yg, dtype=np.float64)
        if xg.shape != yg.shape or xg.ndim != 2:
            raise ValueError("xg, yg must be 2-D arrays of the same shape")
        imax, jmax = xg.shape
        outs = [np.zeros(imax * jmax) for _ in range(10)]
        st = self.lib.v2d_oracle_compute_metrics(imax, jmax, float(dksi), float(deta),
                                                 _ptr(xg), _ptr(yg), *[_ptr(o) for o in outs])
        if st != 0:
            raise ValueError(f"compute_metrics: bad arguments (status {st})")
        return tuple(outs)

    # vorti2d_core.f90:392-495 ; f2py: compute_metrics_local(il0, il1, dksi, deta, xgl, ygl)
    def compute_metrics_local(self, il0, il1, dksi, deta, xgl, ygl):
        xgl = np.asfortranarray(xgl, dtype=np.float64)
        ygl = np.asfortranarray(ygl, dtype=np.float64)
        gxm, jmax = xgl.shape
        outs = [np.zeros(gxm * jmax) for _ in range(10)]
        st = self.lib.v2d_oracle_compute_metrics_local(gxm, jmax, int(il0), int(il1),
                                                       float(dksi), float(deta), _ptr(xgl),
                                                       _ptr(ygl), *[_ptr(o) for o in outs])
        if st != 0:
            raise ValueError(f"compute_metrics_local: bad arguments (status {st})")
        return tuple(outs)

    # vorti2d_core.f90:219-383
    def assemble_coo(self, imax, jmax, re, invdtau, inv2dt, urot, dksi, deta,
                     jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys, yphys,
                     psi, ome, omeold, omeoldold, r0, r1, maxnnz, ff_bc, ca, sa):
        arrs = [_f64(a) for a in (jac, alfa, beta, gama, pmet, qmet, detadx, detady,
                                  xphys, yphys, psi, ome, omeold, omeoldold)]
        ci = np.zeros(maxnnz, dtype=np.intc)
        cj = np.zeros(maxnnz, dtype=np.intc)
        cv = np.zeros(maxnnz)
        bvec = np.zeros(r1 - r0)
        nnz = ctypes.c_int(0)
        st = self.lib.v2d_oracle_assemble_coo(
            int(imax), int(jmax), float(re), float(invdtau), float(inv2dt), float(urot),
            float(dksi), float(deta), *[_ptr(a) for a in arrs], int(r0), int(r1), int(maxnnz),
            int(ff_bc), float(ca), float(sa), _ptr(ci, _ip), _ptr(cj, _ip), _ptr(cv),
            ctypes.byref(nnz), _ptr(bvec))
        if st != 0:
            raise ValueError(f"assemble_coo: status {st} (capacity {maxnnz})")
        return ci, cj, cv, nnz.value, bvec

    # vorti2d_core.f90:510-661
    def assemble_coo_local(self, gxm, jmax, il0, il1, re, invdtau, inv2dt, urot, dksi, deta,
                           jac, alfa, beta, gama, pmet, qmet, detadx, detady, xphys, yphys,
                           psi, ome, omeold, omeoldold, r0, nloc, lg, maxnnz, ff_bc, ca, sa):
        arrs = [_f64(a) for a in (jac, alfa, beta, gama, pmet, qmet, detadx, detady,
                                  xphys, yphys, psi, ome, omeold, omeoldold)]
        lg = np.ascontiguousarray(lg, dtype=np.intc)
        ci = np.zeros(maxnnz, dtype=np.intc)
        cj = np.zeros(maxnnz, dtype=np.intc)
        cv = np.zeros(maxnnz)
        bvec = np.zeros(nloc)
        nnz = ctypes.c_int(0)
        st = self.lib.v2d_oracle_assemble_coo_local(
            int(gxm), int(jmax), int(il0), int(il1), float(re), float(invdtau), float(inv2dt),
            float(urot), float(dksi), float(deta), *[_ptr(a) for a in arrs], int(r0),
            int(nloc), _ptr(lg, _ip), int(maxnnz), int(ff_bc), float(ca), float(sa),
            _ptr(ci, _ip), _ptr(cj, _ip), _ptr(cv), ctypes.byref(nnz), _ptr(bvec))
        if st != 0:
            raise ValueError(f"assemble_coo_local: status {st} (capacity {maxnnz})")
        return ci, cj, cv, nnz.value, bvec


_CORE = None


def core() -> OracleCore:
    global _CORE
    if _CORE is None:
        _CORE = OracleCore()
    return _CORE


# --------------------------------------------------------------------- mesh
def generate_cylinder(imax=181, jmax=181, inner_rad=0.5, outer_rad=50.0):
    """Restates vorti2d/mesh.py:14-50 (radial increments 1,1,1,2,3,...;
    circumferential clustering min(i, imax-i)**0.6; theta = 2 pi (1 - s))."""
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


# ------------------------------------------------------------------- forces
FORCE_COLUMNS = ("t", "cd", "cl", "cm", "cdp", "cdf", "clp", "clf", "cmp", "cmf")


@dataclass
class ForceCoeffs:
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

    def to_dict(self):
        return asdict(self)


def compute_force_coeffs(imax, jmax, re, dksi, deta, beta, gama, detadx, detady,
                         xphys, yphys, ome, ref_length=None, moment_ref=(0.0, 0.0)):
    """Restates vorti2d/forces.py:82-194 (pressure force by parts, friction
    from wall vorticity, P = imax-1 distinct wall nodes)."""
    P = imax - 1
    w = np.arange(P)
    xw, yw, ow = xphys[w], yphys[w], ome[w]
    bw, gw = beta[w], gama[w]
    inv_gn = 1.0 / np.sqrt(bw)
    nx = detadx[w] * inv_gn
    ny = detady[w] * inv_gn
    tx, ty = ny, -nx
    ome_xi = (np.roll(ow, -1) - np.roll(ow, 1)) / (2.0 * dksi)
    ome_eta = (-3.0 * ow + 4.0 * ome[imax + w] - ome[2 * imax + w]) / (2.0 * deta)
    dwdn = (gw * ome_xi + bw * ome_eta) * inv_gn
    seg = np.sqrt((np.roll(xw, -1) - xw) ** 2 + (np.roll(yw, -1) - yw) ** 2)
    ds = 0.5 * (seg + np.roll(seg, 1))
    x0, y0 = moment_ref
    fxp = (1.0 / re) * np.sum(yw * dwdn * ds)
    fyp = -(1.0 / re) * np.sum(xw * dwdn * ds)
    fric = (1.0 / re) * ow
    fxf = np.sum(-fric * tx * ds)
    fyf = np.sum(-fric * ty * ds)
    rx, ry = xw - x0, yw - y0
    mzp = -(1.0 / (2.0 * re)) * np.sum((rx ** 2 + ry ** 2) * dwdn * ds)
    mzf = np.sum((rx * (-fric * ty) - ry * (-fric * tx)) * ds)
    if ref_length is None:
        wsum = ds.sum()
        cx = np.sum(xw * ds) / wsum
        cy = np.sum(yw * ds) / wsum
        ref_length = 2.0 * np.sum(np.sqrt((xw - cx) ** 2 + (yw - cy) ** 2) * ds) / wsum
    d = ref_length
    cdp, cdf = 2.0 * fxp / d, 2.0 * fxf / d
    clp, clf = 2.0 * fyp / d, 2.0 * fyf / d
    cmp_, cmf = 2.0 * mzp / d ** 2, 2.0 * mzf / d ** 2
    return ForceCoeffs(cd=cdp + cdf, cl=clp + clf, cm=cmp_ + cmf, cdp=cdp, cdf=cdf,
                       clp=clp, clf=clf, cmp=cmp_, cmf=cmf, ref_length=d)


# ----------------------------------------------------------------- velocity
def compute_velocity(imax, jmax, dksi, deta, jac, beta, gama, detadx, detady, psi,
                     want_mag=False):
    """Restates vorti2d/velocity.py:38-93: grad(xi) from the exported metrics,
    psi_xi central with the branch-cut wrap, psi_eta central inside and
    one-sided 2nd order at j = 0 and j = jmax-1."""
    xix = (gama * detadx + jac * detady) / beta
    xiy = (gama * detady - jac * detadx) / beta
    p = np.asarray(psi, dtype=np.float64).reshape(jmax, imax)
    i = np.arange(imax)
    e, w = i + 1, i - 1
    e[0] = e[imax - 1] = 1
    w[0] = w[imax - 1] = imax - 2
    pxi = ((p[:, e] - p[:, w]) / (2.0 * dksi)).reshape(-1)
    pe = np.empty_like(p)
    pe[1:-1] = (p[2:] - p[:-2]) / (2.0 * deta)
    pe[0] = (-3.0 * p[0] + 4.0 * p[1] - p[2]) / (2.0 * deta)
    pe[-1] = (3.0 * p[-1] - 4.0 * p[-2] + p[-3]) / (2.0 * deta)
    pe = pe.reshape(-1)
    u = pxi * xiy + pe * detady
    v = -(pxi * xix + pe * detadx)
    if want_mag:
        return u, v, np.sqrt(u * u + v * v)
    return u, v


# ------------------------------------------------------------- config scalars
def config_scalars(re=60.0, steady=False, dt_phys=0.2, dtau=math.inf, alpha_deg=0.0,
                   farfield_bc="dirichlet"):
    """Restates vorti2d/config.py:139-160: (invdtau, inv2dt, ca, sa, ff_bc)."""
    invdtau = 0.0 if math.isinf(dtau) else 1.0 / dtau
    inv2dt = 0.0 if steady else 1.0 / (2.0 * dt_phys)
    codes = {"dirichlet": 0, "outflow": 1, "outflow_psi": 2}
    if farfield_bc.lower() not in codes:
        raise ValueError(f"unknown farfield_bc={farfield_bc!r}")
    a = math.radians(alpha_deg)
    return invdtau, inv2dt, math.cos(a), math.sin(a), codes[farfield_bc.lower()]


def u_rot(t, steady, rot_speed, rot_until):
    """vorti2d/config.py:162-166."""
    if steady:
        return rot_speed
    return rot_speed if t <= rot_until else 0.0


# -------------------------------------------------------------------- solver
def canonical_csr(ci, cj, cv, nrows, ncols):
    """COO -> scipy canonical CSR, as vorti2d/petsc_solver.py:80-89 does."""
    import scipy.sparse as sp
    return sp.csr_matrix((np.asarray(cv, dtype=np.float64),
                          (np.asarray(ci, dtype=np.int64), np.asarray(cj, dtype=np.int64))),
                         shape=(nrows, ncols))


def gmres_ilu_solve(A, b, rtol=1e-10, restart=200, max_it=2000, drop_tol=1e-3, fill_factor=10.0):
    """Stand-in for the reference's iterative CPU solve ``gmres_asm``
    (vorti2d/dist_solver.py:138-158: GMRES(ksp_restart = 200), rtol, at most
    2000 iterations, ASM with ILU(1) subdomain solves -- on one rank the ASM
    subdomain is the whole matrix).  scipy has no level-of-fill ILU, so the
    preconditioner is scipy's threshold ILU (spilu, SuperLU's ILUTP) with the
    given drop tolerance and fill factor and the diagonal as pivot (with
    partial pivoting the incomplete factors of these systems hit exact zero
    pivots).  Returns (x, iterations, converged, relative residual)."""
    import scipy.sparse.linalg as spla
    Ac = A.tocsc()
    ilu = spla.spilu(Ac, drop_tol=drop_tol, fill_factor=fill_factor, diag_pivot_thresh=0.0)
    M = spla.LinearOperator(A.shape, ilu.solve)
    count = [0]

    def cb(_):
        count[0] += 1

    x, info = spla.gmres(A, b, M=M, rtol=rtol, atol=0.0, restart=restart,
                         maxiter=max(1, -(-max_it // restart)), callback=cb,
                         callback_type="pr_norm")
    bn = float(np.linalg.norm(b))
    rel = float(np.linalg.norm(A @ x - b) / bn) if bn > 0 else 0.0
    return x, count[0], info == 0, rel


class OracleSolver:
    """Replicated-path driver restated from vorti2d/solver.py:48-224 (one
    process; MUMPS replaced by scipy SuperLU).  The state arrays and the
    per-step history follow the reference exactly:

    * init (solver.py:103-114): zeros, far-field psi = ca*y - sa*x;
    * Newton (solver.py:117-145): q += dq, res = ||dq||_2 / (2N), loop while
      res > pseudo_tol and it < max_pseudo_iter;
    * time list and BDF2 history shift (solver.py:172-191).
    """

    def __init__(self, xg, yg, re=60.0, steady=False, dt_phys=0.2, t_start=0.0, t_end=50.0,
                 dtau=math.inf, pseudo_tol=1e-10, max_pseudo_iter=200, rot_speed=0.0,
                 rot_until=0.0, farfield_bc="dirichlet", alpha_deg=0.0, linsolve="direct",
                 ref_length=None, moment_center=(0.0, 0.0)):
        self.core = core()
        self.xg, self.yg = np.asarray(xg, dtype=np.float64), np.asarray(yg, dtype=np.float64)
        self.imax, self.jmax = self.xg.shape
        self.ndof = self.imax * self.jmax
        self.dksi = 1.0 / (self.imax - 1)
        self.deta = 1.0 / (self.jmax - 1)
        self.re, self.steady, self.dt_phys = float(re), bool(steady), float(dt_phys)
        self.t_start, self.t_end = float(t_start), float(t_end)
        self.pseudo_tol, self.max_pseudo_iter = float(pseudo_tol), int(max_pseudo_iter)
        self.rot_speed, self.rot_until = float(rot_speed), float(rot_until)
        self.ref_length, self.moment_center = ref_length, moment_center
        self.linsolve = linsolve
        (self.invdtau, self.inv2dt, self.ca, self.sa,
         self.ff_bc) = config_scalars(re, steady, dt_phys, dtau, alpha_deg, farfield_bc)
        (self.jac, self.alfa, self.beta, self.gama, self.pmet, self.qmet, self.detadx,
         self.detady, self.xphys, self.yphys) = self.core.compute_metrics(
            self.dksi, self.deta, self.xg, self.yg)
        self.maxnnz = 2 * self.ndof * 13
        self.psi = np.zeros(self.ndof)
        self.ome = np.zeros(self.ndof)
        self.omeold = np.zeros(self.ndof)
        self.omeoldold = np.zeros(self.ndof)
        ff = slice(self.imax * (self.jmax - 1), self.ndof)
        self.psi[ff] = self.ca * self.yphys[ff] - self.sa * self.xphys[ff]
        self.t = self.t_start
        self.step = 0
        self.history = []          # (t, inner iterations, final res)
        self.n_solves = 0

    def metrics(self):
        return (self.jac, self.alfa, self.beta, self.gama, self.pmet, self.qmet,
                self.detadx, self.detady, self.xphys, self.yphys)

    def assemble(self, urot):
        return self.core.assemble_coo(
            self.imax, self.jmax, self.re, self.invdtau, self.inv2dt, urot, self.dksi,
            self.deta, *self.metrics(), self.psi, self.ome, self.omeold, self.omeoldold,
            0, 2 * self.ndof, self.maxnnz, self.ff_bc, self.ca, self.sa)

    def newton_once(self, urot):
        import scipy.sparse.linalg as spla
        ci, cj, cv, nnz, b = self.assemble(urot)
        A = canonical_csr(ci[:nnz], cj[:nnz], cv[:nnz], 2 * self.ndof, 2 * self.ndof)
        sol = spla.spsolve(A.tocsc(), b)
        self.n_solves += 1
        self.psi += sol[:self.ndof]
        self.ome += sol[self.ndof:]
        return float(np.linalg.norm(sol) / (2.0 * self.ndof))

    def pseudo_solve(self, urot):
        res, it = 1.0e5, 0
        while res > self.pseudo_tol and it < self.max_pseudo_iter:
            res = self.newton_once(urot)
            it += 1
        return res, it

    def times(self):
        if self.steady:
            return [self.t_start]
        nsteps = int(round((self.t_end - self.t_start) / self.dt_phys)) + 1
        return [self.t_start + m * self.dt_phys for m in range(max(nsteps, 0))]

    def advance(self, t):
        """One physical step at time t (solver.py:182-191)."""
        res, it = self.pseudo_solve(u_rot(t, self.steady, self.rot_speed, self.rot_until))
        if not self.steady:
            self.omeoldold = self.omeold.copy()
            self.omeold = self.ome.copy()
        self.t = t
        self.step += 1
        self.history.append((t, it, res))
        return res, it

    def run(self, max_steps=None):
        for m, t in enumerate(self.times()):
            if max_steps is not None and m >= max_steps:
                break
            self.advance(t)
        return self

    def force_coeffs(self):
        return compute_force_coeffs(self.imax, self.jmax, self.re, self.dksi, self.deta,
                                    self.beta, self.gama, self.detadx, self.detady,
                                    self.xphys, self.yphys, self.ome,
                                    ref_length=self.ref_length,
                                    moment_ref=self.moment_center)
