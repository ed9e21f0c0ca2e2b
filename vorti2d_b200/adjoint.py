"""Discrete adjoint of the steady solve: gradients of the force coefficients
(Cl, Cd, Cm) with respect to the angle of attack and the Reynolds number,
exposed as a ``torch.autograd.Function``.

At a converged steady state R(q; p) = 0 (R = -b, the residual whose exact
Jacobian J = dR/dq the Newton iteration assembles), a force coefficient
C(q; p) has

    dC/dp = dC/dp|_q - lambda^T dR/dp|_q,      J^T lambda = (dC/dq)^T.

* dC/dq: the coefficients are linear in the vorticity at the wall rows
  (vorti2d/forces.py:82-194: wall-normal vorticity gradient and wall
  friction), so their gradient is formed exactly by ``force_gradients``.
* lambda: one transposed solve per vector-Jacobian product, on the device
  (``v2d_solver_adjoint``: FP64 multifrontal factors of J, transposed solve,
  refinement against J^T products).
* dR/dRe: R is affine in 1/Re, so two residual evaluations give it exactly;
  dC/dRe|_q = -C/Re because every force term carries 1/Re.
* dR/dalpha: the far-field streamfunction rows (psi = cos(a) y - sin(a) x),
  by a central difference of the residual (alpha in degrees).  The forces are
  body-axis quantities, so dC/dalpha|_q = 0.  With an outflow far field the
  set of outflow rows itself depends on alpha; gradients in alpha are for the
  Dirichlet far field.
* Shape: the P = imax-1 distinct wall nodes move along their outward normals
  by d_i, and each grid line follows with a weight that decays from 1 at the
  wall to 0 at the far field (``deform_ogrid``; linear in d).  dR/dd_i and
  dC/dd_i|_q are forward-mode (tangent) derivatives through the metric
  computation, the residual rows and the wall force integrals on the device
  (``v2d_solver_shape_tangent``: dual numbers, one CTA per direction, only
  the four grid lines a direction touches): exact, with no step size.  The
  one adjoint solve is shared by all P components.  Central differences on
  displaced meshes (``v2d_solver_shape_gradient``) remain available as a
  check (``method="fd"``).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check, dptr, lib


def force_gradients(imax, jmax, re, dksi, deta, beta, gama, detadx, detady, xphys, yphys,
                    ref_length=None, moment_ref=(0.0, 0.0)):
    """d(Cd, Cl, Cm)/d(omega) at every node (three arrays of imax*jmax), for
    the force integrals of vorti2d/forces.py:82-194 (P = imax-1 distinct wall
    nodes; periodic-central omega_xi and one-sided omega_eta at the wall)."""
    N = imax * jmax
    P = imax - 1
    w = np.arange(P)
    wp, wm = (w + 1) % P, (w - 1) % P
    xw, yw = xphys[w], yphys[w]
    bw, gw = beta[w], gama[w]
    inv_gn = 1.0 / np.sqrt(bw)
    nx, ny = detadx[w] * inv_gn, detady[w] * inv_gn
    tx, ty = ny, -nx
    seg = np.sqrt((xw[wp] - xw) ** 2 + (yw[wp] - yw) ** 2)
    ds = 0.5 * (seg + seg[wm])
    if ref_length is None:
        wsum = ds.sum()
        cx, cy = np.sum(xw * ds) / wsum, np.sum(yw * ds) / wsum
        ref_length = 2.0 * np.sum(np.sqrt((xw - cx) ** 2 + (yw - cy) ** 2) * ds) / wsum
    d = float(ref_length)
    rx, ry = xw - moment_ref[0], yw - moment_ref[1]
    # C = sum_w a_w dwdn_w + sum_w c_w omega_w
    terms = {
        "cd": ((2.0 / d) * (1.0 / re) * yw * ds, (2.0 / d) * (-1.0 / re) * tx * ds),
        "cl": (-(2.0 / d) * (1.0 / re) * xw * ds, (2.0 / d) * (-1.0 / re) * ty * ds),
        "cm": (-(2.0 / d ** 2) * (1.0 / (2.0 * re)) * (rx ** 2 + ry ** 2) * ds,
               (2.0 / d ** 2) * (1.0 / re) * (-rx * ty + ry * tx) * ds),
    }
    out = {}
    for key, (a, c) in terms.items():
        g = np.zeros(N)
        k = a * inv_gn
        np.add.at(g, wp, k * gw / (2.0 * dksi))
        np.add.at(g, wm, -k * gw / (2.0 * dksi))
        np.add.at(g, w, k * bw * (-3.0) / (2.0 * deta) + c)
        np.add.at(g, imax + w, k * bw * 4.0 / (2.0 * deta))
        np.add.at(g, 2 * imax + w, k * bw * (-1.0) / (2.0 * deta))
        out[key] = g
    return out


def _residual(solver, re, alpha_deg, urot):
    cfg = solver.cfg
    a = math.radians(alpha_deg)
    b = np.empty(2 * solver.ndof)
    check(lib().v2d_solver_residual(solver.dev.h, float(re), cfg.inv_dtau(), cfg.inv_2dt(),
                                    float(urot), math.cos(a), math.sin(a), dptr(b)),
          "residual")
    return b


def adjoint_solve(solver, g, rtol=1e-10, max_refine=20):
    """lambda with J^T lambda = g at the solver's current state."""
    g = np.ascontiguousarray(g, dtype=np.float64)
    lam = np.empty_like(g)
    its, rel = ctypes.c_int(), ctypes.c_double()
    urot = solver.cfg.u_rot(solver.t)
    check(lib().v2d_solver_adjoint(solver.dev.h, float(urot), dptr(g), dptr(lam), float(rtol),
                                   int(max_refine), ctypes.byref(its), ctypes.byref(rel)),
          "adjoint")
    return lam, its.value, rel.value


def force_vjp(solver, weights, alpha_h=1e-3):
    """d(w . (Cl, Cd, Cm))/d(alpha_deg, Re) at the solver's converged steady
    state, for output weights w = (w_cl, w_cd, w_cm)."""
    cfg = solver.cfg
    re, adeg = float(cfg.re), float(cfg.alpha_deg)
    urot = cfg.u_rot(solver.t)
    grads = force_gradients(solver.imax, solver.jmax, re, solver.dksi, solver.deta, solver.beta,
                            solver.gama, solver.detadx, solver.detady, solver.xphys,
                            solver.yphys, cfg.ref_length, cfg.moment_center)
    w_cl, w_cd, w_cm = (float(v) for v in weights)
    N = solver.ndof
    g = np.zeros(2 * N)
    g[N:] = w_cl * grads["cl"] + w_cd * grads["cd"] + w_cm * grads["cm"]
    fc = solver.force_coeffs()
    lam, its, rel = adjoint_solve(solver, g)
    # dR/dRe (affine in 1/Re): b(s) = A + B s, dC/dRe = dC/dRe|q + lambda^T db/dRe
    b1, b2 = _residual(solver, re, adeg, urot), _residual(solver, 2.0 * re, adeg, urot)
    db_ds = (b1 - b2) / (1.0 / re - 0.5 / re)
    db_dre = db_ds * (-1.0 / re ** 2)
    dC_dre_q = -(w_cl * fc.cl + w_cd * fc.cd + w_cm * fc.cm) / re
    d_re = dC_dre_q + float(lam @ db_dre)
    bp, bm = _residual(solver, re, adeg + alpha_h, urot), _residual(solver, re, adeg - alpha_h, urot)
    d_alpha = float(lam @ ((bp - bm) / (2.0 * alpha_h)))
    return d_alpha, d_re, dict(refinements=its, rel_res=rel)


# ------------------------------------------------------------------ shape
def steady_solve_ser(solver, dtau0=1.0, tol=None, max_iter=300, dtau_max=1e12, growth=2.0,
                     reject=1e3, re=None):
    """Steady state by pseudo-transient continuation: iteration k adds
    1/dtau_k to the Newton Jacobian's diagonal.  While the residual norm
    ||R|| falls, dtau grows by `growth` per iteration, and at least to the
    switched-evolution-relaxation value dtau0 ||R_0|| / ||R_k|| (Mulder and
    van Leer, 1985); a step that raises ||R|| more than `reject` times, or
    fails, is undone (the previous state is restored) and dtau shrinks
    fourfold; a step that raises it less halves dtau (the residual may rise
    for a while on the way; only blow-ups are undone).  dtau stays within
    [dtau0 / 64, dtau_max].  The first iterations are damped pseudo-time
    steps, the last ones Newton steps.  The residual carries no pseudo-time
    term, so the fixed point is the steady solution of the reference's
    equations; the stopping rule is the reference's, ||dq||/(2N) <= tol.
    For cases where Newton from the free stream diverges.  Returns
    (||dq||/(2N), iterations, counting rejected ones); the handle's own
    1/dtau is restored.  `re`: the Reynolds number the handle currently
    solves for, when it was changed from the configuration's (continuation
    in Re)."""
    dev, cfg = solver.dev, solver.cfg
    tol = cfg.pseudo_tol if tol is None else float(tol)
    urot = cfg.u_rot(0.0)
    re = float(cfg.re) if re is None else float(re)
    adeg = float(cfg.alpha_deg)
    keep = dev.params.invdtau
    r0 = float(np.linalg.norm(_residual(solver, re, adeg, urot)))
    r_prev = r0
    res, it, dtau = math.inf, 0, float(dtau0)
    dmin = float(dtau0) / 64.0
    try:
        while res > tol and it < max_iter:
            saved = [a.copy() for a in dev.get_state()]
            dev.set_invdtau(1.0 / dtau)
            code, res, _ = dev.newton(urot)
            solver._host_state = None
            it += 1
            ok = code in (_lib.V2D_OK, _lib.V2D_ENOTCONVERGED) and math.isfinite(res)
            rk = float(np.linalg.norm(_residual(solver, re, adeg, urot))) if ok else math.inf
            if not (ok and math.isfinite(rk)) or rk > reject * r_prev:
                dev.set_state(*saved)       # undo the step
                solver._host_state = None
                res = math.inf              # the undone step's update norm is no result
                if dtau <= dmin:
                    break
                dtau = max(dmin, 0.25 * dtau)
                continue
            if rk < r_prev:
                dtau = min(dtau_max, max(dtau * growth, dtau0 * r0 / max(rk, 1e-300)))
            else:
                dtau = max(dmin, 0.5 * dtau)
            r_prev = rk
    finally:
        dev.set_invdtau(keep)
    return res, it


def wall_normals(xg, yg):
    """Outward unit normals (nx, ny) of the P = imax-1 distinct wall nodes
    (j = 0) of an O-grid (xg, yg of shape (imax, jmax)), from the periodic
    central tangent, pointing toward the first grid line off the wall."""
    xg, yg = np.asarray(xg, dtype=np.float64), np.asarray(yg, dtype=np.float64)
    P = xg.shape[0] - 1
    xw, yw = xg[:P, 0], yg[:P, 0]
    tx = np.roll(xw, -1) - np.roll(xw, 1)
    ty = np.roll(yw, -1) - np.roll(yw, 1)
    tn = np.hypot(tx, ty)
    nx, ny = ty / tn, -tx / tn
    sgn = np.where(nx * (xg[:P, 1] - xw) + ny * (yg[:P, 1] - yw) < 0.0, -1.0, 1.0)
    return nx * sgn, ny * sgn


def deformation_weights(xg, yg):
    """phi (imax, jmax): (1 - w)^2 with w the arclength fraction along each
    grid line from the wall (1 at the wall, 0 at the far field)."""
    xg, yg = np.asarray(xg, dtype=np.float64), np.asarray(yg, dtype=np.float64)
    seg = np.hypot(np.diff(xg, axis=1), np.diff(yg, axis=1))
    cum = np.concatenate([np.zeros((xg.shape[0], 1)), np.cumsum(seg, axis=1)], axis=1)
    w = cum / cum[:, -1:]
    return (1.0 - w) ** 2


def deform_ogrid(xg, yg, d, normals=None, weights=None):
    """The O-grid with wall node i moved by d[i] along its outward normal and
    grid line i by d[i] * phi[i, j] (the seam column imax-1 moves with
    column 0).
    ``normals`` / ``weights`` default to those of (xg, yg), so the map is
    linear in d."""
    xg, yg = np.asarray(xg, dtype=np.float64), np.asarray(yg, dtype=np.float64)
    P = xg.shape[0] - 1
    d = np.asarray(d, dtype=np.float64)
    if d.shape != (P,):
        raise ValueError(f"d must have imax-1 = {P} entries (got shape {d.shape})")
    nx, ny = normals if normals is not None else wall_normals(xg, yg)
    phi = weights if weights is not None else deformation_weights(xg, yg)
    X, Y = xg.copy(), yg.copy()
    X[:P] += (d * nx)[:, None] * phi[:P]
    Y[:P] += (d * ny)[:, None] * phi[:P]
    X[P] += d[0] * nx[0] * phi[P]
    Y[P] += d[0] * ny[0] * phi[P]
    return X, Y


def gaussian_bumps(P, n_bumps=8, amplitude=1e-3, width=None, seed=0):
    """A seeded wall displacement: n_bumps periodic Gaussian bumps over the P
    wall nodes, centres uniform, signs random, each of height ``amplitude``
    and standard deviation ``width`` nodes (default P/32)."""
    rng = np.random.default_rng(seed)
    sigma = float(width) if width is not None else P / 32.0
    centres = rng.uniform(0.0, P, n_bumps)
    signs = rng.choice([-1.0, 1.0], n_bumps)
    i = np.arange(P, dtype=np.float64)
    d = np.zeros(P)
    for c, sg in zip(centres, signs):
        dist = np.abs(i - c)
        dist = np.minimum(dist, P - dist)
        d += sg * amplitude * np.exp(-0.5 * (dist / sigma) ** 2)
    return d


def residual_on_mesh(solver, xg, yg, met_rows=3):
    """(b, wall metrics): b = -R at the solver's state with the metrics of
    mesh (xg, yg), and rows j < met_rows of the 10 metric arrays, shape
    (10, met_rows * imax)."""
    cfg = solver.cfg
    X = np.asfortranarray(xg, dtype=np.float64)
    Y = np.asfortranarray(yg, dtype=np.float64)
    if X.shape != (solver.imax, solver.jmax) or Y.shape != X.shape:
        raise ValueError(f"mesh must be {solver.imax} x {solver.jmax}")
    b = np.empty(2 * solver.ndof)
    met = np.empty((10, met_rows * solver.imax))
    a = math.radians(cfg.alpha_deg)
    check(lib().v2d_solver_residual_mesh(solver.dev.h, dptr(X), dptr(Y), float(cfg.re),
                                         cfg.inv_dtau(), cfg.inv_2dt(),
                                         float(cfg.u_rot(solver.t)), math.cos(a), math.sin(a),
                                         dptr(b), int(met_rows), dptr(met)),
          "residual_mesh")
    return b, met


def _wall_forces(solver, met3, ome3, weights):
    from .forces import compute_force_coeffs
    cfg = solver.cfg
    fc = compute_force_coeffs(solver.imax, 3, float(cfg.re), solver.dksi, solver.deta,
                              met3[2], met3[3], met3[6], met3[7], met3[8], met3[9], ome3,
                              ref_length=cfg.ref_length, moment_ref=cfg.moment_center)
    w_cl, w_cd, w_cm = (float(v) for v in weights)
    return w_cl * fc.cl + w_cd * fc.cd + w_cm * fc.cm


def shape_vjp(solver, weights, base_mesh, h=None, method="tangent"):
    """d(w . (Cl, Cd, Cm))/d(d_i), i < P, at the solver's converged steady
    state, for wall displacements d along the normals of ``base_mesh`` (the
    undeformed (xg, yg) that ``deform_ogrid`` displaced to the solver's
    mesh), with one adjoint solve.  method "tangent": exact tangent
    derivatives of the residual and the force integrals on the device
    (``v2d_solver_shape_tangent``); "fd": central differences of step h
    (default 1e-6 of the wall's extent) on the 2P displaced meshes
    (``v2d_solver_shape_gradient``)."""
    if method not in ("tangent", "fd"):
        raise ValueError(f"unknown method {method!r}")
    xg0, yg0 = (np.asarray(a, dtype=np.float64) for a in base_mesh)
    nx, ny = wall_normals(xg0, yg0)
    phi = np.asfortranarray(deformation_weights(xg0, yg0))
    X = np.asarray(solver.xg, dtype=np.float64)
    Y = np.asarray(solver.yg, dtype=np.float64)
    P = solver.imax - 1
    if h is None and method == "fd":
        h = 1e-6 * max(np.ptp(X[:P, 0]), np.ptp(Y[:P, 0]))
    cfg = solver.cfg
    grads = force_gradients(solver.imax, solver.jmax, float(cfg.re), solver.dksi, solver.deta,
                            solver.beta, solver.gama, solver.detadx, solver.detady,
                            solver.xphys, solver.yphys, cfg.ref_length, cfg.moment_center)
    w_cl, w_cd, w_cm = (float(v) for v in weights)
    N = solver.ndof
    g = np.zeros(2 * N)
    g[N:] = w_cl * grads["cl"] + w_cd * grads["cd"] + w_cm * grads["cm"]
    lam, its, rel = adjoint_solve(solver, g)
    nx = np.ascontiguousarray(nx)
    ny = np.ascontiguousarray(ny)
    dots = np.empty(P)
    a = math.radians(cfg.alpha_deg)
    rl = -1.0 if cfg.ref_length is None else float(cfg.ref_length)
    mc = cfg.moment_center
    if method == "tangent":
        dforces = np.empty((P, 10))
        check(lib().v2d_solver_shape_tangent(solver.dev.h, dptr(nx), dptr(ny), dptr(phi),
                                             dptr(lam), float(cfg.re), cfg.inv_dtau(),
                                             cfg.inv_2dt(), float(cfg.u_rot(solver.t)),
                                             math.cos(a), math.sin(a), rl, float(mc[0]),
                                             float(mc[1]), dptr(dots), dptr(dforces)),
              "shape_tangent")
        # v2d_force_coeffs order: cd, cl, cm, ...
        dc = w_cd * dforces[:, 0] + w_cl * dforces[:, 1] + w_cm * dforces[:, 2]
        return dc + dots, dict(refinements=its, rel_res=rel, method="tangent")
    forces = np.empty((P, 2, 10))
    check(lib().v2d_solver_shape_gradient(solver.dev.h, dptr(nx), dptr(ny), dptr(phi), dptr(lam),
                                          float(h), float(cfg.re), cfg.inv_dtau(), cfg.inv_2dt(),
                                          float(cfg.u_rot(solver.t)), math.cos(a), math.sin(a),
                                          rl, float(mc[0]), float(mc[1]), dptr(dots),
                                          dptr(forces)),
          "shape_gradient")
    # v2d_force_coeffs order: cd, cl, cm, ...
    c = w_cd * forces[:, :, 0] + w_cl * forces[:, :, 1] + w_cm * forces[:, :, 2]
    out = (c[:, 0] - c[:, 1]) / (2.0 * h) + dots / (2.0 * h)
    return out, dict(refinements=its, rel_res=rel, h=h, method="fd")


def _torch():
    import torch
    return torch


class SteadyForces:
    """(alpha_deg, Re[, wall displacements d]) -> (Cl, Cd, Cm) of a converged
    steady solve, as a torch.autograd.Function whose backward is the
    discrete adjoint.

    Usage::

        out = SteadyForces.apply(alpha, re, make_solver)   # out = [Cl, Cd, Cm]
        out = SteadyForces.apply(alpha, re, make_solver, d, base_mesh)

    ``make_solver(alpha_deg, re)`` -- or ``make_solver(alpha_deg, re, d)``
    when a displacement tensor d (P = imax-1 entries) is given -- returns a
    ``vorti2d_b200.Solver`` configured as a steady case, on
    ``deform_ogrid(*base_mesh, d)`` in the second form; it is advanced once
    (the steady Newton solve) and kept for the backward pass.
    """

    _fn = None

    @classmethod
    def function(cls):
        if cls._fn is None:
            torch = _torch()

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, alpha, re, make_solver, disp, base_mesh):
                    if disp is None:
                        s = make_solver(float(alpha), float(re))
                    else:
                        s = make_solver(float(alpha), float(re),
                                        disp.detach().cpu().numpy().astype(np.float64))
                    s.advance(s.times()[0])
                    fc = s.force_coeffs()
                    ctx.solver = s
                    ctx.base_mesh = base_mesh
                    ctx.has_disp = disp is not None
                    return torch.tensor([fc.cl, fc.cd, fc.cm], dtype=torch.float64)

                @staticmethod
                def backward(ctx, grad):
                    s = ctx.solver
                    w = grad.detach().cpu().numpy()
                    d_alpha, d_re, _ = force_vjp(s, w)
                    d_disp = None
                    if ctx.has_disp:
                        gs, _ = shape_vjp(s, w, ctx.base_mesh)
                        d_disp = torch.tensor(gs, dtype=torch.float64)
                    s.close()
                    return (torch.tensor(d_alpha, dtype=torch.float64),
                            torch.tensor(d_re, dtype=torch.float64), None, d_disp, None)

            cls._fn = _Fn
        return cls._fn

    @classmethod
    def apply(cls, alpha, re, make_solver, disp=None, base_mesh=None):
        if disp is not None and base_mesh is None:
            raise ValueError("a displacement needs the undeformed base_mesh")
        return cls.function().apply(alpha, re, make_solver, disp, base_mesh)
