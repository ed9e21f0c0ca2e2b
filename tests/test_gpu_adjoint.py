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
    # GMRES on J^T, preconditioned by the transposed solve of FP64 factors
    assert np.linalg.norm(J.T @ lam - g) <= 1e-10 * np.linalg.norm(g), (its, rel)
    assert its <= 6
    s.close()


def test_transposed_solve_wide_fronts(v2d, oracle_mod):
    """257x257 unsteady cylinder after one BDF2 step (separators of up to 514
    unknowns): J^T lambda = g to 1e-10 through GMRES on J^T with the
    transposed multifrontal solve as its preconditioner."""
    from vorti2d_b200.adjoint import adjoint_solve
    xg, yg = oracle_mod.generate_cylinder(257, 257)
    cfg = v2d.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                     re=200.0, steady=False, dt_phys=0.05, farfield_bc="outflow",
                     pseudo_tol=1e-12, max_pseudo_iter=8, ksp_rtol=1e-12, precision="fp64")
    s = v2d.Solver(cfg, mesh=(xg, yg))
    s.advance(s.times()[0])
    g = np.random.default_rng(1).standard_normal(2 * s.ndof)
    lam, its, rel = adjoint_solve(s, g, rtol=1e-10)
    ip, ix, dv, _ = s.dev.system(urot=cfg.u_rot(0.0))
    J = sp.csr_matrix((dv, ix, ip), shape=(2 * s.ndof, 2 * s.ndof))
    assert np.linalg.norm(J.T @ lam - g) <= 2e-10 * np.linalg.norm(g), (its, rel)
    s.close()


def test_ser_continuation_reaches_the_newton_state(v2d, oracle_mod):
    """steady_solve_ser (pseudo-time steps whose dtau grows as the update
    norm falls) ends on the state plain Newton reaches: the fixed point
    carries no pseudo-time term."""
    from vorti2d_b200.adjoint import steady_solve_ser
    xg, yg = oracle_mod.generate_cylinder(IMAX, JMAX)
    ref = solve(v2d, xg, yg, RE, ADEG)
    s = v2d.Solver(steady_cfg(v2d, RE, ADEG), mesh=(xg, yg))
    res, its = steady_solve_ser(s, dtau0=0.5, max_iter=120)
    assert res <= 1e-13 and its > 0, (res, its)
    for a, b in ((s.psi, ref.psi), (s.ome, ref.ome)):
        assert np.max(np.abs(a - b)) <= 1e-9 * max(1.0, np.max(np.abs(b)))
    assert abs(s.force_coeffs().cd - ref.force_coeffs().cd) <= 1e-10
    assert s.dev.params.invdtau == 0.0
    ref.close()
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


def test_residual_on_own_mesh_is_the_handles(v2d, oracle_mod):
    """The residual and metrics on a given mesh equal the handle's own when
    that mesh is the handle's, bit for bit; the wall force integral from the
    three returned rows equals the solver's force coefficients."""
    from vorti2d_b200.adjoint import _residual, _wall_forces, residual_on_mesh
    xg, yg = oracle_mod.generate_cylinder(33, 25)
    s = solve(v2d, xg, yg, RE, ADEG)
    b, met = residual_on_mesh(s, xg, yg, 3)
    want = _residual(s, RE, ADEG, s.cfg.u_rot(s.t))
    assert np.array_equal(b, want)
    own = s.dev.metrics()
    for q in range(10):
        assert np.array_equal(met[q], own[q][:3 * s.imax]), q
    ome3 = s.ome[:3 * s.imax]
    for w, key in (((1, 0, 0), "cl"), ((0, 1, 0), "cd"), ((0, 0, 1), "cm")):
        got = _wall_forces(s, met, ome3, w)
        ref = getattr(s.force_coeffs(), key)
        assert abs(got - ref) <= 1e-14 * max(1.0, abs(ref)), key
    s.close()


SHAPE_CASES = [
    # (kind, imax, jmax, Re, alpha, ref_length)
    ("cylinder", 65, 49, 40.0, 4.0, None),
    ("naca", 65, 33, 5.0, 3.0, 1.0),
]


def _base_mesh(v2d, oracle_mod, kind, im, jm):
    if kind == "cylinder":
        return oracle_mod.generate_cylinder(im, jm)
    return v2d.generate_naca0012(im, jm)


def _shape_solve(v2d, base, d, re, adeg, ref_length):
    from vorti2d_b200.adjoint import deform_ogrid
    X, Y = deform_ogrid(*base, d)
    cfg = steady_cfg(v2d, re, adeg)
    cfg.ref_length = ref_length
    s = v2d.Solver(cfg, mesh=(X, Y))
    s.advance(0.0)
    return s


@pytest.mark.parametrize("kind,im,jm,re,adeg,ref_length", SHAPE_CASES)
def test_shape_gradient_matches_finite_differences(v2d, oracle_mod, kind, im, jm, re, adeg,
                                                   ref_length):
    """dCl/dd and dCd/dd for the wall-normal displacements d of all P wall
    nodes (one adjoint solve) against central differences of full steady
    solves along a bump direction and a single-node direction, on the GPU
    and on the oracle, within 1e-5 relative."""
    from vorti2d_b200.adjoint import deform_ogrid, gaussian_bumps, shape_vjp
    base = _base_mesh(v2d, oracle_mod, kind, im, jm)
    P = im - 1
    d0 = gaussian_bumps(P, n_bumps=4, amplitude=1e-3, seed=1)
    s = _shape_solve(v2d, base, d0, re, adeg, ref_length)
    grads = {}
    for w, key in (((1.0, 0.0, 0.0), "cl"), ((0.0, 1.0, 0.0), "cd")):
        grads[key], info = shape_vjp(s, w, base)
        assert grads[key].shape == (P,)
    s.close()
    e5 = np.zeros(P)
    e5[5] = 1.0
    # steps small enough that the O(eps^2) error of the full-solve difference
    # is below 1e-7 relative: moving one wall node by 1e-4 is a sizeable part
    # of the local cell there
    for v, eps in ((gaussian_bumps(P, n_bumps=3, amplitude=1.0, seed=2), 1e-5), (e5, 1e-6)):
        fd, fo = {}, {}
        sp_ = _shape_solve(v2d, base, d0 + eps * v, re, adeg, ref_length)
        sm_ = _shape_solve(v2d, base, d0 - eps * v, re, adeg, ref_length)
        for key in ("cl", "cd"):
            fd[key] = (getattr(sp_.force_coeffs(), key) - getattr(sm_.force_coeffs(), key)) / (2 * eps)
        sp_.close()
        sm_.close()
        ov = []
        for sg in (1.0, -1.0):
            X, Y = deform_ogrid(*base, d0 + sg * eps * v)
            o = oracle_mod.OracleSolver(X, Y, re=re, alpha_deg=adeg, steady=True,
                                        pseudo_tol=1e-13, max_pseudo_iter=60).run()
            ov.append(oracle_mod.compute_force_coeffs(
                o.imax, o.jmax, o.re, o.dksi, o.deta, o.beta, o.gama, o.detadx, o.detady,
                o.xphys, o.yphys, o.ome, ref_length=ref_length))
        for key in ("cl", "cd"):
            fo[key] = (getattr(ov[0], key) - getattr(ov[1], key)) / (2 * eps)
            adj = float(grads[key] @ v)
            scale = max(abs(fd[key]), 1e-3 * np.abs(grads[key]).sum())
            assert abs(adj - fd[key]) <= 1e-5 * scale, (kind, key, adj, fd[key])
            assert abs(adj - fo[key]) <= 1e-5 * scale, (kind, key, adj, fo[key])


def test_torch_autograd_shape(v2d, oracle_mod):
    import torch
    from vorti2d_b200.adjoint import SteadyForces, deform_ogrid, gaussian_bumps, shape_vjp
    base = oracle_mod.generate_cylinder(33, 25)
    P = 32
    d0 = gaussian_bumps(P, n_bumps=3, amplitude=1e-3, seed=4)

    def make(adeg, re, d):
        return v2d.Solver(steady_cfg(v2d, re, adeg), mesh=deform_ogrid(*base, d))

    alpha = torch.tensor(ADEG, dtype=torch.float64, requires_grad=True)
    re = torch.tensor(RE, dtype=torch.float64, requires_grad=True)
    d = torch.tensor(d0, dtype=torch.float64, requires_grad=True)
    out = SteadyForces.apply(alpha, re, make, d, base)
    out[1].backward()
    s = make(ADEG, RE, d0)
    s.advance(0.0)
    want, _ = shape_vjp(s, (0.0, 1.0, 0.0), base)
    s.close()
    assert d.grad is not None and d.grad.shape == (P,)
    assert np.allclose(d.grad.numpy(), want, rtol=1e-10, atol=1e-12 * np.abs(want).max())
    assert alpha.grad is not None and re.grad is not None


def test_device_shape_gradient_equals_host_route(v2d, oracle_mod):
    """The device loop over the 2P displaced meshes (v2d_solver_shape_gradient)
    gives the same components as the host route through residual_on_mesh and
    the wall force integral, for the seam node, an interior node and the last
    node."""
    from vorti2d_b200.adjoint import (_wall_forces, adjoint_solve, deform_ogrid,
                                      deformation_weights, force_gradients, gaussian_bumps,
                                      residual_on_mesh, shape_vjp, wall_normals)
    base = oracle_mod.generate_cylinder(33, 25)
    P = 32
    d0 = gaussian_bumps(P, n_bumps=3, amplitude=1e-3, seed=5)
    X, Y = deform_ogrid(*base, d0)
    s = v2d.Solver(steady_cfg(v2d, RE, ADEG), mesh=(X, Y))
    s.advance(0.0)
    w = (0.3, 1.0, -0.2)
    h = 1e-6
    dev, _ = shape_vjp(s, w, base, h=h, method="fd")
    nx, ny = wall_normals(*base)
    phi = deformation_weights(*base)
    grads = force_gradients(s.imax, s.jmax, RE, s.dksi, s.deta, s.beta, s.gama, s.detadx,
                            s.detady, s.xphys, s.yphys)
    g = np.zeros(2 * s.ndof)
    g[s.ndof:] = w[0] * grads["cl"] + w[1] * grads["cd"] + w[2] * grads["cm"]
    lam, _, _ = adjoint_solve(s, g)
    ome3 = s.ome[:3 * s.imax]
    for i in (0, 7, P - 1):
        vals, bs = [], []
        for sg in (1.0, -1.0):
            Xs, Ys = X.copy(), Y.copy()
            Xs[i] += sg * h * nx[i] * phi[i]
            Ys[i] += sg * h * ny[i] * phi[i]
            if i == 0:
                Xs[P] += sg * h * nx[0] * phi[P]
                Ys[P] += sg * h * ny[0] * phi[P]
            b, met = residual_on_mesh(s, Xs, Ys, 3)
            bs.append(b)
            vals.append(_wall_forces(s, met, ome3, w))
        host = (vals[0] - vals[1]) / (2 * h) + float(lam @ (bs[0] - bs[1])) / (2 * h)
        assert abs(dev[i] - host) <= 1e-8 * max(1.0, abs(host)), (i, dev[i], host)
    s.close()


@pytest.mark.parametrize("kind,im,jm,re,adeg,ref_length", SHAPE_CASES)
def test_shape_tangent_equals_extrapolated_differences(v2d, oracle_mod, kind, im, jm, re, adeg,
                                                       ref_length):
    """The exact tangent shape gradient (dual numbers through metrics,
    residual and wall integrals) against the displaced-mesh central
    differences extrapolated in the step (Richardson over h, h/2, h/4: error
    O(h^6)), for every wall node at once, within 1e-8 relative to the
    gradient's largest component."""
    from vorti2d_b200.adjoint import deform_ogrid, gaussian_bumps, shape_vjp
    base = _base_mesh(v2d, oracle_mod, kind, im, jm)
    P = im - 1
    d0 = gaussian_bumps(P, n_bumps=4, amplitude=1e-3, seed=3)
    s = _shape_solve(v2d, base, d0, re, adeg, ref_length)
    w = (0.7, 1.0, -0.4)
    tan, info = shape_vjp(s, w, base)
    assert info["method"] == "tangent"
    h = 1e-4 * max(np.ptp(base[0][:P, 0]), np.ptp(base[1][:P, 0]))
    f1, _ = shape_vjp(s, w, base, h=h, method="fd")
    f2, _ = shape_vjp(s, w, base, h=h / 2, method="fd")
    f4, _ = shape_vjp(s, w, base, h=h / 4, method="fd")
    r1, r2 = (4.0 * f2 - f1) / 3.0, (4.0 * f4 - f2) / 3.0
    rich = (16.0 * r2 - r1) / 15.0
    scale = np.abs(tan).max()
    err = np.abs(tan - rich).max() / scale
    print(f"{kind}: tangent vs extrapolated differences, max rel {err:.2e} "
          f"(plain h={h:.1e}: {np.abs(tan - f1).max() / scale:.2e}, once extrapolated: "
          f"{np.abs(tan - r2).max() / scale:.2e})")
    assert err <= 1e-8, err
    s.close()
