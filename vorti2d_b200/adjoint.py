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


def _torch():
    import torch
    return torch


class SteadyForces:
    """(alpha_deg, Re) -> (Cl, Cd, Cm) of a converged steady solve, as a
    torch.autograd.Function whose backward is the discrete adjoint.

    Usage::

        out = SteadyForces.apply(alpha, re, make_solver)   # out = [Cl, Cd, Cm]

    ``make_solver(alpha_deg, re)`` returns a ``vorti2d_b200.Solver`` configured
    as a steady case; it is advanced once (the steady Newton solve) and kept
    for the backward pass.
    """

    _fn = None

    @classmethod
    def function(cls):
        if cls._fn is None:
            torch = _torch()

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, alpha, re, make_solver):
                    s = make_solver(float(alpha), float(re))
                    s.advance(s.times()[0])
                    fc = s.force_coeffs()
                    ctx.solver = s
                    return torch.tensor([fc.cl, fc.cd, fc.cm], dtype=torch.float64)

                @staticmethod
                def backward(ctx, grad):
                    s = ctx.solver
                    d_alpha, d_re, _ = force_vjp(s, grad.detach().cpu().numpy())
                    s.close()
                    return (torch.tensor(d_alpha, dtype=torch.float64),
                            torch.tensor(d_re, dtype=torch.float64), None)

            cls._fn = _Fn
        return cls._fn

    @classmethod
    def apply(cls, alpha, re, make_solver):
        return cls.function().apply(alpha, re, make_solver)
