"""Converged Newton / BDF2 solves on the GPU against the oracle's direct
(SuperLU) solves: psi/omega within 1e-9, force coefficients within 1e-8, plus
the reference's boundary-value checks (tests/test_smoke.py:44-56,
tests/test_postproc.py:121-142)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    return np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b)))


def gpu_cfg(v2d, **kw):
    base = dict(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                ksp_restart=100, ksp_rtol=1e-12, krylov_max_it=20000, pseudo_tol=1e-12,
                max_pseudo_iter=30)
    base.update(kw)
    return v2d.Config(**base)


def test_unsteady_bdf2_matches_oracle(v2d, oracle_mod):
    imax = jmax = 33
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    kw = dict(re=100.0, steady=False, dt_phys=0.2, rot_speed=0.5, rot_until=2.0,
              farfield_bc="outflow")
    ref = oracle_mod.OracleSolver(xg, yg, pseudo_tol=1e-12, max_pseudo_iter=30, **kw)
    s = v2d.Solver(gpu_cfg(v2d, **kw), mesh=(xg, yg))
    for t in ref.times()[:4]:
        ref.advance(t)
        s.advance(t)
        assert _close(s.psi, ref.psi, 1e-9)
        assert _close(s.ome, ref.ome, 1e-9)
        assert _close(s.omeold, ref.omeold, 1e-9)
    fg, fo = s.force_coeffs(), ref.force_coeffs()
    for k in ("cd", "cl", "cm"):
        assert abs(getattr(fg, k) - getattr(fo, k)) <= 1e-8
    s.close()


def test_steady_newton_matches_oracle(v2d, oracle_mod):
    """Steady Re=20, pure Newton (dtau = inf) on a 17x17 O-grid (where the
    oracle's Newton converges in 8 iterations): GMRES(256) with block Jacobi
    against the oracle's direct solves; then the reference's boundary-value
    and symmetry checks (tests/test_smoke.py:44-56)."""
    imax, jmax = 17, 17
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    ref = oracle_mod.OracleSolver(xg, yg, re=20.0, steady=True, pseudo_tol=1e-13,
                                  max_pseudo_iter=50).run()
    assert ref.history[-1][2] < 1e-13
    s = v2d.Solver(gpu_cfg(v2d, re=20.0, steady=True, ksp_restart=256, krylov_max_it=100000,
                           pseudo_tol=1e-13, max_pseudo_iter=50, precond="bjacobi"),
                   mesh=(xg, yg))
    s.advance(0.0)
    dpsi = np.max(np.abs(s.psi - ref.psi))
    dome = np.max(np.abs(s.ome - ref.ome))
    assert _close(s.psi, ref.psi, 1e-9), (dpsi, s.newton_log)
    assert _close(s.ome, ref.ome, 1e-9), (dome, s.newton_log)
    fg, fo = s.force_coeffs(), ref.force_coeffs()
    assert abs(fg.cd - fo.cd) <= 1e-8 and abs(fg.cl - fo.cl) <= 1e-8
    N = imax * jmax
    ff = slice(imax * (jmax - 1), N)
    assert np.max(np.abs(s.psi[ff] - s.yphys[ff])) < 1e-10
    assert np.max(np.abs(s.psi[:imax])) < 1e-10
    assert np.max(np.abs(s.ome[ff])) < 1e-12
    assert abs(s.psi.max() + s.psi.min()) < 1e-6
    s.close()


def test_mixed_precision_matches_fp64(v2d, oracle_mod):
    """FP32 Krylov inside FP64 defect correction converges to the FP64
    solution: |dCd| < 1e-6 and fields within 1e-9 after 3 BDF2 steps."""
    imax = jmax = 33
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    kw = dict(re=100.0, steady=False, dt_phys=0.2, rot_speed=0.5, rot_until=2.0,
              farfield_bc="outflow")
    a = v2d.Solver(gpu_cfg(v2d, **kw), mesh=(xg, yg))
    b = v2d.Solver(gpu_cfg(v2d, precision="mixed", **kw), mesh=(xg, yg))
    for t in a.times()[:3]:
        a.advance(t)
        b.advance(t)
    assert abs(a.force_coeffs().cd - b.force_coeffs().cd) < 1e-6
    assert _close(b.psi, a.psi, 1e-9) and _close(b.ome, a.ome, 1e-9)
    a.close()
    b.close()


def test_angle_of_attack_far_field(v2d, oracle_mod):
    """alpha rotates the free stream: far-field psi = cos(a) y - sin(a) x
    (tests/test_postproc.py:121-142)."""
    imax = jmax = 25
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    s = v2d.Solver(gpu_cfg(v2d, re=20.0, steady=False, dt_phys=0.2, alpha_deg=12.0),
                   mesh=(xg, yg))
    s.advance(0.0)
    ff = slice(imax * (jmax - 1), imax * jmax)
    c, sn = np.cos(np.radians(12.0)), np.sin(np.radians(12.0))
    assert np.max(np.abs(s.psi[ff] - (c * s.yphys[ff] - sn * s.xphys[ff]))) < 1e-9
    s.close()


def test_run_writes_reference_formats(v2d, oracle_mod, tmp_path):
    """run() writes forces.csv (header + one row per step) and a restart .npz
    in the reference's format; resuming continues at t + dt
    (tests/test_smoke.py:59-74)."""
    xg, yg = oracle_mod.generate_cylinder(25, 17)
    v2d.save_mesh(xg, yg, str(tmp_path / "xg.csv"), str(tmp_path / "yg.csv"))
    kw = dict(re=40.0, steady=False, dt_phys=0.5, rot_speed=0.5, rot_until=2.0,
              mesh_xg=str(tmp_path / "xg.csv"), mesh_yg=str(tmp_path / "yg.csv"),
              out_dir=str(tmp_path / "out"), restart_out="r.npz", compute_forces=True)
    s = v2d.run(gpu_cfg(v2d, t_end=1.0, **kw))
    rows = open(tmp_path / "out" / "forces.csv").read().strip().splitlines()
    assert rows[0].startswith("t,cd,cl,cm") and len(rows) == 1 + 3
    r = np.load(tmp_path / "out" / "r.npz")
    assert set(r.files) >= {"psi", "ome", "omeold", "omeoldold", "t", "step", "imax", "jmax", "re"}
    cfg2 = gpu_cfg(v2d, t_end=1.5, **kw)
    cfg2.restart_in = str(tmp_path / "out" / "r.npz")
    s2 = v2d.run(cfg2)
    assert abs(s2.t - 1.5) < 1e-12
    s.close()
    s2.close()
