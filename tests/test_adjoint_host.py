"""Host-side pieces of the adjoint: the force-coefficient gradient with
respect to the vorticity is exact, because the integrals of
vorti2d/forces.py:82-194 are linear in omega (checked against the oracle's
restatement of that module)."""
import numpy as np
import pytest


@pytest.mark.parametrize("ref_length,mref", [(None, (0.0, 0.0)), (1.0, (0.25, -0.1))])
def test_force_gradient_is_the_linear_functional(oracle_mod, ref_length, mref):
    from vorti2d_b200.adjoint import force_gradients
    imax, jmax = 33, 21
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    dk, de = 1 / (imax - 1), 1 / (jmax - 1)
    M = oracle_mod.core().compute_metrics(dk, de, xg, yg)
    args = (imax, jmax, 40.0, dk, de, M[2], M[3], M[6], M[7], M[8], M[9])
    g = force_gradients(*args, ref_length=ref_length, moment_ref=mref)
    rng = np.random.default_rng(3)
    for _ in range(3):
        ome = rng.standard_normal(imax * jmax)
        fc = oracle_mod.compute_force_coeffs(*args, ome, ref_length=ref_length, moment_ref=mref)
        for k in ("cd", "cl", "cm"):
            want = getattr(fc, k)
            assert abs(g[k] @ ome - want) <= 1e-12 * max(1.0, abs(want)), k


def _cyl(oracle_mod, im=33, jm=25):
    return oracle_mod.generate_cylinder(im, jm)


def test_wall_normals_are_outward_unit_vectors(oracle_mod):
    from vorti2d_b200.adjoint import wall_normals
    xg, yg = _cyl(oracle_mod)
    nx, ny = wall_normals(xg, yg)
    P = xg.shape[0] - 1
    assert nx.shape == (P,)
    assert np.allclose(np.hypot(nx, ny), 1.0, atol=1e-14)
    # the cylinder is centred at the origin: outward = along the position
    assert np.all(nx * xg[:P, 0] + ny * yg[:P, 0] > 0.99 * np.hypot(xg[:P, 0], yg[:P, 0]))


def test_deform_ogrid_is_linear_and_keeps_far_field_and_seam(oracle_mod):
    from vorti2d_b200.adjoint import deform_ogrid, gaussian_bumps, wall_normals
    xg, yg = _cyl(oracle_mod)
    P = xg.shape[0] - 1
    X0, Y0 = deform_ogrid(xg, yg, np.zeros(P))
    assert np.array_equal(X0, xg) and np.array_equal(Y0, yg)
    d1 = gaussian_bumps(P, n_bumps=3, amplitude=1e-3, seed=1)
    d2 = gaussian_bumps(P, n_bumps=5, amplitude=2e-3, seed=2)
    X1, Y1 = deform_ogrid(xg, yg, d1)
    X2, Y2 = deform_ogrid(xg, yg, d2)
    X12, Y12 = deform_ogrid(xg, yg, d1 + d2)
    assert np.allclose(X12 - xg, (X1 - xg) + (X2 - xg), atol=1e-13, rtol=0)
    assert np.allclose(Y12 - yg, (Y1 - yg) + (Y2 - yg), atol=1e-13, rtol=0)
    assert np.array_equal(X1[:, -1], xg[:, -1]) and np.array_equal(Y1[:, -1], yg[:, -1])
    assert np.allclose(X1[-1] - xg[-1], X1[0] - xg[0], atol=1e-18)
    assert np.allclose(Y1[-1] - yg[-1], Y1[0] - yg[0], atol=1e-18)
    nx, ny = wall_normals(xg, yg)
    assert np.allclose(X1[:P, 0] - xg[:P, 0], d1 * nx, atol=1e-16)
    assert np.allclose(Y1[:P, 0] - yg[:P, 0], d1 * ny, atol=1e-16)
    with pytest.raises(ValueError):
        deform_ogrid(xg, yg, np.zeros(P + 1))


def test_gaussian_bumps_are_seeded_and_bounded():
    from vorti2d_b200.adjoint import gaussian_bumps
    a, b = gaussian_bumps(256, seed=7), gaussian_bumps(256, seed=7)
    assert np.array_equal(a, b) and a.shape == (256,)
    assert not np.array_equal(a, gaussian_bumps(256, seed=8))
    assert 0.0 < np.abs(a).max() <= 8 * 1e-3
    # periodic: the bumps wrap around the seam without a jump
    assert abs(a[0] - a[-1]) < 0.2 * 1e-3


def test_steady_forces_needs_base_mesh_with_displacement():
    torch = pytest.importorskip("torch")
    from vorti2d_b200.adjoint import SteadyForces
    with pytest.raises(ValueError):
        SteadyForces.apply(torch.tensor(0.0), torch.tensor(40.0), None, torch.zeros(4))


def test_unsteady_adjoint_history_rows():
    from vorti2d_b200.unsteady_adjoint import _interior_ome_rows
    rows = _interior_ome_rows(5, 4)
    # 2N = 40 unknowns; the BDF2 history sits on the vorticity rows of j = 1, 2
    assert list(rows) == list(range(20 + 5, 20 + 15))
