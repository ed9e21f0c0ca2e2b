"""Discrete adjoint of the unsteady BDF2 run: the gradient of the time-mean
of w . (Cl, Cd, Cm) over the run's steps with respect to the angle of attack
and the Reynolds number, with checkpoints and recomputation.

Each step n solves R_n(q_n; omega_{n-1}, omega_{n-2}; p) = 0 by Newton
(vorti2d/solver.py:136-191).  The BDF2 history enters the right-hand side
b = -R only on the interior vorticity rows, as
-(3 omega - 4 omega^n + omega^{n-1}) inv2dt (vorti2d_core.f90:376-377), so
db_{n+1}/d omega_n = +4 inv2dt and db_{n+2}/d omega_n = -inv2dt there.  For
J = (1/M) sum_n C_n(q_n) the adjoint runs backward in time:

    J_n^T lambda_n = (dC_n/dq_n)^T / M + (db_{n+1}/dq_n)^T lambda_{n+1}
                                       + (db_{n+2}/dq_n)^T lambda_{n+2},
    dJ/dp = sum_n lambda_n . db_n/dp + (1/M) sum_n dC_n/dp|_q.

J_n is the Newton Jacobian at step n's converged state (v2d_solver_adjoint
assembles and factors it in FP64 and solves the transposed system).  The
states come from checkpoints taken every ``checkpoint_every`` steps of the
forward run: each segment is recomputed forward from its checkpoint, its
converged states kept, and then swept backward.  The exact adjoint needs
every step converged to the tolerance of the comparison (pseudo_tol well
below the Newton default), since the discrete equations it differentiates
are the converged ones.  The initial vorticity (zero) does not depend on
(alpha, Re).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check, dptr, lib
from .adjoint import _residual, force_gradients


def _coeffs(fc):
    return np.array([fc.cl, fc.cd, fc.cm])


def _interior_ome_rows(imax, jmax):
    """Indices (into the 2N system) of the vorticity rows that carry the BDF2
    history term: 1 <= j <= jmax-2, every i."""
    N = imax * jmax
    k = np.arange(imax, (jmax - 1) * imax)
    return N + k


def _adjoint(solver, urot, g, rtol=1e-10, max_refine=20):
    lam = np.empty_like(g)
    its, rel = ctypes.c_int(), ctypes.c_double()
    check(lib().v2d_solver_adjoint(solver.dev.h, float(urot), dptr(g), dptr(lam), float(rtol),
                                   int(max_refine), ctypes.byref(its), ctypes.byref(rel)),
          "adjoint")
    return lam


def unsteady_mean_force_vjp(make_solver, n_steps, weights, checkpoint_every=20, alpha_h=1e-3):
    """(J, dJ/dalpha_deg, dJ/dRe, info) for J = mean over the first n_steps
    BDF2 steps of w . (Cl, Cd, Cm), w = weights.

    ``make_solver()`` returns a fresh unsteady ``vorti2d_b200.Solver`` at its
    initial state.  The forward run keeps a checkpoint of the state every
    ``checkpoint_every`` steps; the backward sweep recomputes one segment at
    a time from its checkpoint."""
    w = np.asarray(weights, dtype=np.float64)
    s = make_solver()
    cfg = s.cfg
    if cfg.steady:
        raise ValueError("the unsteady adjoint needs an unsteady configuration")
    times = s.times()[:n_steps]
    M = len(times)
    if M == 0:
        raise ValueError("n_steps must be >= 1")
    C = int(checkpoint_every)
    if C < 1:
        raise ValueError("checkpoint_every must be >= 1")
    re, adeg = float(cfg.re), float(cfg.alpha_deg)
    imax, jmax, N = s.imax, s.jmax, s.ndof
    rows = _interior_ome_rows(imax, jmax)
    inv2dt = cfg.inv_2dt()
    # forward: checkpoints and the force coefficients of every step
    ckpt, coeffs = {}, np.empty((M, 3))
    for n, t in enumerate(times):
        if n % C == 0:
            ckpt[n] = [a.copy() for a in s.dev.get_state()]
        s.advance(t)
        coeffs[n] = _coeffs(s.force_coeffs())
    per_step = coeffs @ w                   # w . C_n for every step
    Jval = float(per_step.sum()) / M
    grads = force_gradients(imax, jmax, re, s.dksi, s.deta, s.beta, s.gama, s.detadx, s.detady,
                            s.xphys, s.yphys, cfg.ref_length, cfg.moment_center)
    cq = np.zeros(2 * N)
    cq[N:] = (w[0] * grads["cl"] + w[1] * grads["cd"] + w[2] * grads["cm"]) / M
    d_alpha = 0.0
    d_re = -float(per_step.sum()) / re / M  # every force term carries 1/Re
    lam1 = np.zeros(2 * N)                  # lambda_{n+1}
    lam2 = np.zeros(2 * N)                  # lambda_{n+2}
    solves = 0
    for n0 in sorted(ckpt, reverse=True):
        n1 = min(n0 + C, M)
        s.set_state(*ckpt[n0])
        seg = []
        for n in range(n0, n1):
            before = s.dev.get_state()
            s.advance(times[n])
            after = s.dev.get_state()
            # step n's converged state with its history (before the shift)
            seg.append((after[0].copy(), after[1].copy(), before[2].copy(), before[3].copy()))
        for n in range(n1 - 1, n0 - 1, -1):
            psi, ome, om1, om2 = seg[n - n0]
            s.set_state(psi, ome, om1, om2)
            urot = cfg.u_rot(times[n])
            g = cq.copy()
            g[rows] += 4.0 * inv2dt * lam1[rows] - inv2dt * lam2[rows]
            lam = _adjoint(s, urot, g)
            solves += 1
            b1 = _residual(s, re, adeg, urot)
            b2 = _residual(s, 2.0 * re, adeg, urot)
            db_dre = (b1 - b2) / (1.0 / re - 0.5 / re) * (-1.0 / re ** 2)
            d_re += float(lam @ db_dre)
            bp = _residual(s, re, adeg + alpha_h, urot)
            bm = _residual(s, re, adeg - alpha_h, urot)
            d_alpha += float(lam @ ((bp - bm) / (2.0 * alpha_h)))
            lam2, lam1 = lam1, lam
    s.close()
    return Jval, d_alpha, d_re, dict(steps=M, checkpoints=len(ckpt), adjoint_solves=solves)


class UnsteadyMeanForces:
    """(alpha_deg, Re) -> time-mean (Cl, Cd, Cm) over the first n_steps BDF2
    steps, as a torch.autograd.Function whose backward is the checkpointed
    discrete adjoint (one backward sweep per output weight vector).

    Usage::

        out = UnsteadyMeanForces.apply(alpha, re, make_solver, n_steps, checkpoint_every)

    ``make_solver(alpha_deg, re)`` returns a fresh unsteady
    ``vorti2d_b200.Solver`` at its initial state.
    """

    _fn = None

    @classmethod
    def function(cls):
        if cls._fn is None:
            import torch

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, alpha, re, make_solver, n_steps, checkpoint_every):
                    a, r = float(alpha), float(re)
                    s = make_solver(a, r)
                    acc = np.zeros(3)
                    times = s.times()[:n_steps]
                    for t in times:
                        s.advance(t)
                        acc += _coeffs(s.force_coeffs())
                    s.close()
                    ctx.args = (a, r, make_solver, n_steps, checkpoint_every)
                    return torch.tensor(acc / max(len(times), 1), dtype=torch.float64)

                @staticmethod
                def backward(ctx, grad):
                    a, r, make_solver, n_steps, every = ctx.args
                    w = grad.detach().cpu().numpy().astype(np.float64)
                    _, d_alpha, d_re, _ = unsteady_mean_force_vjp(
                        lambda: make_solver(a, r), n_steps, w, checkpoint_every=every)
                    return (torch.tensor(d_alpha, dtype=torch.float64),
                            torch.tensor(d_re, dtype=torch.float64), None, None, None)

            cls._fn = _Fn
        return cls._fn

    @classmethod
    def apply(cls, alpha, re, make_solver, n_steps, checkpoint_every=20):
        return cls.function().apply(alpha, re, make_solver, int(n_steps), int(checkpoint_every))
