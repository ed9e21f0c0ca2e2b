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
