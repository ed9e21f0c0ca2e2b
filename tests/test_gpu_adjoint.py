"""Discrete adjoint of the steady solve on the GPU: the transposed
multifrontal solve satisfies J^T lambda = g, and the adjoint gradients of
(Cl, Cd, Cm) with respect to (alpha, Re) agree with central finite
differences of the steady solve (the GPU's and the oracle's) within 1e-5
relative."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

IMAX, JMAX = 65, 49
RE, ADEG = 40.0, 4.0


def steady_cfg(v2d, re, adeg):
    return v2d.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                      re=re, alpha_deg=adeg, steady=True, pseudo_tol=1e-13, max_pseudo_iter=60,
                      ksp_rtol=1e-12)


def solve(v2d, xg, yg, re, adeg):
    s = v2d.Solver(steady_cfg(v2d, re, adeg), mesh=(xg, yg))
    s.advance(0.0)
    return s


def coeffs(fc):
    return np.array([fc.cl, fc.cd, fc.cm])


def test_transposed_solve(v2d, oracle_mod):
    from vorti2d_b200.adjoint import adjoint_solve
    xg, yg = oracle_mod.generate_cylinder(33, 25)
    s = solve(v2d, xg, yg, RE, ADEG)
    g = np.random.default_rng(0).standard_normal(2 * s.ndof)
    lam, its, rel = adjoint_solve(s, g, rtol=1e-12)
    ip, ix, dv, _ = s.dev.system(urot=0.0)
    J = sp.csr_matrix((dv, ix, ip), shape=(2 * s.ndof, 2 * s.ndof))
    # refinement stops at the attainable accuracy of the FP64 factors
    assert np.linalg.norm(J.T @ lam - g) <= 1e-10 * np.linalg.norm(g), (its, rel)
    assert its <= 6
    s.close()


def test_adjoint_gradients_match_finite_differences(v2d, oracle_mod):
    from vorti2d_b200.adjoint import force_vjp
    xg, yg = oracle_mod.generate_cylinder(IMAX, JMAX)
    s = solve(v2d, xg, yg, RE, ADEG)
    jac = np.zeros((3, 2))
    for i in range(3):
        w = np.zeros(3)
        w[i] = 1.0
        d_alpha, d_re, info = force_vjp(s, w)
        jac[i] = d_alpha, d_re
    s.close()
    ha, hr = 1e-3, 1e-3 * RE
    fd = np.zeros((3, 2))
    fo = np.zeros((3, 2))
    for col, (da, dr, h) in enumerate([(ha, 0.0, ha), (0.0, hr, hr)]):
        cp = solve(v2d, xg, yg, RE + dr, ADEG + da)
        cm = solve(v2d, xg, yg, RE - dr, ADEG - da)
        fd[:, col] = (coeffs(cp.force_coeffs()) - coeffs(cm.force_coeffs())) / (2 * h)
        cp.close()
        cm.close()
        op = oracle_mod.OracleSolver(xg, yg, re=RE + dr, alpha_deg=ADEG + da, steady=True,
                                     pseudo_tol=1e-13, max_pseudo_iter=60).run()
        om = oracle_mod.OracleSolver(xg, yg, re=RE - dr, alpha_deg=ADEG - da, steady=True,
                                     pseudo_tol=1e-13, max_pseudo_iter=60).run()
        fo[:, col] = (coeffs(op.force_coeffs()) - coeffs(om.force_coeffs())) / (2 * h)
    scale = np.abs(fd).max(axis=0)      # per parameter
    assert np.all(np.abs(jac - fd) <= 1e-5 * scale), (jac, fd)
    assert np.all(np.abs(jac - fo) <= 1e-5 * scale), (jac, fo)
    assert abs(jac[0, 0]) > 1e-3       # Cl responds to the angle of attack


def test_torch_autograd_function(v2d, oracle_mod):
    import torch
    from vorti2d_b200.adjoint import SteadyForces, force_vjp
    xg, yg = oracle_mod.generate_cylinder(33, 25)

    def make(adeg, re):
        return v2d.Solver(steady_cfg(v2d, re, adeg), mesh=(xg, yg))

    alpha = torch.tensor(ADEG, dtype=torch.float64, requires_grad=True)
    re = torch.tensor(RE, dtype=torch.float64, requires_grad=True)
    out = SteadyForces.apply(alpha, re, make)
    loss = 2.0 * out[0] + out[1] - 0.5 * out[2]
    loss.backward()
    s = solve(v2d, xg, yg, RE, ADEG)
    d_alpha, d_re, _ = force_vjp(s, np.array([2.0, 1.0, -0.5]))
    s.close()
    assert abs(alpha.grad.item() - d_alpha) <= 1e-10 * max(1.0, abs(d_alpha))
    assert abs(re.grad.item() - d_re) <= 1e-10 * max(1.0, abs(d_re))
    assert np.allclose(out.detach().numpy(),
                       coeffs(solve(v2d, xg, yg, RE, ADEG).force_coeffs()), rtol=1e-12)
