"""Discrete adjoint of the unsteady BDF2 run with checkpoints: the gradient
of the time-mean of w . (Cl, Cd, Cm) with respect to (alpha, Re) agrees with
central differences of complete unsteady runs, and does not depend on the
checkpoint spacing."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RE, ADEG, STEPS = 100.0, 4.0, 7
W = (1.0, 0.5, -0.3)


def _cfg(v2d, re, adeg):
    return v2d.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                      re=re, alpha_deg=adeg, steady=False, dt_phys=0.2, rot_speed=0.5,
                      rot_until=0.6, farfield_bc="dirichlet", pseudo_tol=1e-13,
                      max_pseudo_iter=30, ksp_rtol=1e-12, precision="fp64")


def _mean(v2d, mesh, re, adeg):
    s = v2d.Solver(_cfg(v2d, re, adeg), mesh=mesh)
    acc = 0.0
    for t in s.times()[:STEPS]:
        s.advance(t)
        fc = s.force_coeffs()
        acc += W[0] * fc.cl + W[1] * fc.cd + W[2] * fc.cm
    s.close()
    return acc / STEPS


def test_unsteady_adjoint_matches_finite_differences(v2d, oracle_mod):
    from vorti2d_b200.unsteady_adjoint import unsteady_mean_force_vjp
    mesh = oracle_mod.generate_cylinder(33, 25)
    J, d_alpha, d_re, info = unsteady_mean_force_vjp(
        lambda: v2d.Solver(_cfg(v2d, RE, ADEG), mesh=mesh), STEPS, W, checkpoint_every=3)
    assert info["steps"] == STEPS and info["checkpoints"] == 3
    assert info["adjoint_solves"] == STEPS
    assert abs(J - _mean(v2d, mesh, RE, ADEG)) <= 1e-12 * max(1.0, abs(J))
    ha, hr = 1e-3, 1e-3 * RE
    fd_a = (_mean(v2d, mesh, RE, ADEG + ha) - _mean(v2d, mesh, RE, ADEG - ha)) / (2 * ha)
    fd_r = (_mean(v2d, mesh, RE + hr, ADEG) - _mean(v2d, mesh, RE - hr, ADEG)) / (2 * hr)
    assert abs(d_alpha - fd_a) <= 1e-5 * max(abs(fd_a), 1e-6), (d_alpha, fd_a)
    assert abs(d_re - fd_r) <= 1e-5 * max(abs(fd_r), 1e-6), (d_re, fd_r)
    assert abs(fd_a) > 1e-4 and abs(fd_r) > 1e-6


def test_checkpoint_spacing_does_not_change_the_gradient(v2d, oracle_mod):
    from vorti2d_b200.unsteady_adjoint import unsteady_mean_force_vjp
    mesh = oracle_mod.generate_cylinder(33, 25)
    out = []
    for every in (1, 4, STEPS):
        J, da, dr, info = unsteady_mean_force_vjp(
            lambda: v2d.Solver(_cfg(v2d, RE, ADEG), mesh=mesh), STEPS, W, checkpoint_every=every)
        assert info["checkpoints"] == -(-STEPS // every)
        out.append((J, da, dr))
    for J, da, dr in out[1:]:
        assert abs(J - out[0][0]) <= 1e-12 * max(1.0, abs(J))
        assert abs(da - out[0][1]) <= 1e-8 * max(1.0, abs(da))
        assert abs(dr - out[0][2]) <= 1e-8 * max(1.0, abs(dr))


def test_torch_autograd_unsteady(v2d, oracle_mod):
    import torch
    from vorti2d_b200.unsteady_adjoint import UnsteadyMeanForces, unsteady_mean_force_vjp
    mesh = oracle_mod.generate_cylinder(33, 25)

    def make(adeg, re):
        return v2d.Solver(_cfg(v2d, re, adeg), mesh=mesh)

    alpha = torch.tensor(ADEG, dtype=torch.float64, requires_grad=True)
    re = torch.tensor(RE, dtype=torch.float64, requires_grad=True)
    out = UnsteadyMeanForces.apply(alpha, re, make, STEPS, 3)
    loss = W[0] * out[0] + W[1] * out[1] + W[2] * out[2]
    assert abs(loss.item() - _mean(v2d, mesh, RE, ADEG)) <= 1e-12 * max(1.0, abs(loss.item()))
    loss.backward()
    J, da, dr, _ = unsteady_mean_force_vjp(lambda: make(ADEG, RE), STEPS, W, checkpoint_every=3)
    assert abs(alpha.grad.item() - da) <= 1e-10 * max(1.0, abs(da))
    assert abs(re.grad.item() - dr) <= 1e-10 * max(1.0, abs(dr))
