"""Velocity reconstruction on the device (vorti2d/velocity.py:76-93) against
golden vectors made by the reference's own velocity.py, and the reference's
physical checks of it on a steady solve (tests/test_postproc.py:40-59)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "reference_golden.npz")


@pytest.mark.parametrize("mesh", ["25x17", "65x49"])
def test_velocity_kernel_bit_exact(v2d, mesh):
    golden = np.load(GOLDEN)
    im, jm = (int(v) for v in mesh.split("x"))
    key = f"velocity_{mesh}"
    g = {n: golden[f"{key}_in_{n}"] for n in ("jac", "beta", "gama", "detadx", "detady", "psi")}
    u, v, mag = v2d.compute_velocity(im, jm, 1.0 / (im - 1), 1.0 / (jm - 1), g["jac"], g["beta"],
                                     g["gama"], g["detadx"], g["detady"], g["psi"], want_mag=True)
    want = golden[f"{key}_out"]
    assert np.array_equal(u, want[0]) and np.array_equal(v, want[1])
    assert np.array_equal(mag, want[2])
    u2, v2 = v2d.compute_velocity(im, jm, 1.0 / (im - 1), 1.0 / (jm - 1), g["jac"], g["beta"],
                                  g["gama"], g["detadx"], g["detady"], g["psi"])
    assert np.array_equal(u2, u) and np.array_equal(v2, v)


def test_velocity_of_steady_solutions(v2d, oracle_mod):
    """tests/test_postproc.py:40-59 on the GPU solver (121x121, Re=20): no slip
    at the fixed wall, u -> 1 in the far field, |V| = rot_speed on a rotating
    wall; the solver-state entry point equals the host-array one."""
    xg, yg = oracle_mod.generate_cylinder(121, 121)
    kw = dict(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
              re=20.0, steady=True, pseudo_tol=1e-11, max_pseudo_iter=80, ksp_rtol=1e-10)
    imax = jmax = 121
    wall = slice(0, imax)
    ff = slice(imax * (jmax - 1), imax * jmax)
    s = v2d.Solver(v2d.Config(**kw), mesh=(xg, yg))
    s.advance(0.0)
    u, vv, mag = s.velocity(want_mag=True)
    assert np.abs(u[wall]).max() < 5e-3 and np.abs(vv[wall]).max() < 5e-3
    assert abs(u[ff].mean() - 1.0) < 0.02
    assert np.allclose(mag, np.sqrt(u ** 2 + vv ** 2))
    hu, hv = v2d.compute_velocity(s.imax, s.jmax, s.dksi, s.deta, s.jac, s.beta, s.gama,
                                  s.detadx, s.detady, s.psi)
    assert np.array_equal(hu, u) and np.array_equal(hv, vv)
    s.close()
    sr = v2d.Solver(v2d.Config(rot_speed=0.5, **kw), mesh=(xg, yg))
    sr.advance(0.0)
    _, _, magr = sr.velocity(want_mag=True)
    assert abs(magr[wall].mean() - 0.5) < 0.02
    sr.close()
