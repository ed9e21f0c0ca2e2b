"""The oracle against the reference's own known-answer tests.

The reference's Fortran core and PETSc/MUMPS layer cannot be built here, so
the restatement is pinned by the checks the reference's tests make on that
path (tests/test_smoke.py, tests/test_postproc.py, tests/test_metrics_local.py,
tests/test_assemble_local.py) plus the drag values its documentation records
(docs/verification.rst:132-147).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from cases import local_layout, smooth_state, to_local


def steady(O, imax, jmax, re, inner=0.5, outer=50.0, **kw):
    xg, yg = O.generate_cylinder(imax, jmax, inner, outer)
    kw.setdefault("pseudo_tol", 1e-11)
    kw.setdefault("max_pseudo_iter", 80)
    return O.OracleSolver(xg, yg, re=re, steady=True, **kw).run()


def test_metrics_finite(oracle_mod):
    """tests/test_smoke.py:37-41."""
    xg, yg = oracle_mod.generate_cylinder(31, 31, 0.5, 50.0)
    for a in oracle_mod.core().compute_metrics(1 / 30, 1 / 30, xg, yg):
        assert np.isfinite(a).all()


def test_nnz_formula(oracle_mod):
    """nnz(ff_bc=0) = 23*imax*(jmax-2) + 7*imax (vorti2d_core.f90:247-381:
    psi interior 10, ome interior 13, wall 1 + 4, far field 1 + 1)."""
    for imax, jmax in [(9, 7), (33, 21), (129, 129)]:
        xg, yg = oracle_mod.generate_cylinder(imax, jmax)
        M = oracle_mod.core().compute_metrics(1 / (imax - 1), 1 / (jmax - 1), xg, yg)
        N = imax * jmax
        z = np.zeros(N)
        *_, nnz, _ = oracle_mod.core().assemble_coo(
            imax, jmax, 40.0, 0, 0, 0, 1 / (imax - 1), 1 / (jmax - 1), *M, z, z, z, z, 0,
            2 * N, 26 * N, 0, 1.0, 0.0)
        assert nnz == 23 * imax * (jmax - 2) + 7 * imax


def test_steady_converges_and_bcs(oracle_mod):
    """tests/test_smoke.py:44-56: steady Re=40 on 41x41."""
    s = steady(oracle_mod, 41, 41, 40.0, pseudo_tol=1e-10, max_pseudo_iter=50)
    imax, jmax = s.imax, s.jmax
    ff = slice(imax * (jmax - 1), imax * jmax)
    wall = slice(0, imax)
    assert s.history[-1][2] <= 1e-10
    assert np.max(np.abs(s.psi[ff] - s.yphys[ff])) < 1e-10
    assert np.max(np.abs(s.psi[wall])) < 1e-10
    assert np.max(np.abs(s.ome[ff])) < 1e-12
    assert abs(s.psi.max() + s.psi.min()) < 1e-6


def test_metrics_local_equals_global(oracle_mod):
    """tests/test_metrics_local.py:18-56 (33x21, owned columns, 1e-10)."""
    imax, jmax = 33, 21
    ni, gxs, gxm, il0, il1, gc, lg = local_layout(imax, jmax)
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    dk, de = 1 / (imax - 1), 1 / (jmax - 1)
    G = oracle_mod.core().compute_metrics(dk, de, xg, yg)
    L = oracle_mod.core().compute_metrics_local(il0, il1, dk, de, xg[:ni][gc], yg[:ni][gc])
    for g, loc in zip(G[:8], L[:8]):
        g2 = g.reshape(jmax, imax)[:, :ni]
        l2 = loc.reshape(jmax, gxm)[:, il0 - 1:il1]
        assert np.max(np.abs(g2 - l2)) <= 1e-10 * max(1.0, np.max(np.abs(g2)))


def test_assemble_local_equals_global(oracle_mod):
    """tests/test_assemble_local.py:33-99: both orderings of the Newton
    system of the smooth analytic state give the same update per node."""
    imax, jmax = 25, 17
    re, ff_bc, ca, sa = 80.0, 1, 1.0, 0.0
    invdtau, inv2dt, urot = 0.0, 1.0 / (2 * 0.2), 0.3
    dk, de = 1.0 / (imax - 1), 1.0 / (jmax - 1)
    C = oracle_mod.core()
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = C.compute_metrics(dk, de, xg, yg)
    st = smooth_state(M[8], M[9])
    N = imax * jmax
    ci, cj, cv, nnz, b = C.assemble_coo(imax, jmax, re, invdtau, inv2dt, urot, dk, de, *M,
                                        *st, 0, 2 * N, 26 * N, ff_bc, ca, sa)
    A = sp.csr_matrix((cv[:nnz], (ci[:nnz], cj[:nnz])), shape=(2 * N, 2 * N))
    dg = spla.spsolve(A.tocsc(), b)
    ni, gxs, gxm, il0, il1, gc, lg = local_layout(imax, jmax)
    Ml = C.compute_metrics_local(il0, il1, dk, de, xg[:ni][gc], yg[:ni][gc])
    loc = [to_local(f, imax, jmax, gxm, gc) for f in st]
    nloc = 2 * ni * jmax
    li, lj, lv, lnnz, lb = C.assemble_coo_local(gxm, jmax, il0, il1, re, invdtau, inv2dt,
                                                urot, dk, de, *Ml, *loc, 0, nloc, lg,
                                                14 * nloc, ff_bc, ca, sa)
    Al = sp.csr_matrix((lv[:lnnz], (li[:lnnz], lj[:lnnz])), shape=(nloc, nloc))
    dl = spla.spsolve(Al.tocsc(), lb)
    dpsi_g = dg[:N].reshape(jmax, imax)[:, :ni]
    dome_g = dg[N:].reshape(jmax, imax)[:, :ni]
    dpsi_l = dl[0::2].reshape(jmax, ni)
    dome_l = dl[1::2].reshape(jmax, ni)
    scale = max(np.max(np.abs(dg)), 1.0)
    assert np.max(np.abs(dpsi_g - dpsi_l)) <= 1e-9 * scale
    assert np.max(np.abs(dome_g - dome_l)) <= 1e-9 * scale


@pytest.mark.slow
def test_forces_match_ingham(oracle_mod):
    """tests/test_postproc.py:26-37: steady 121x121, Cd within 5% of Ingham
    (Re=20: 1.998, Re=40: 1.50), no lift or moment, both drag parts > 0."""
    for re, cd_ref in [(20.0, 1.998), (40.0, 1.50)]:
        fc = steady(oracle_mod, 121, 121, re).force_coeffs()
        assert abs(fc.ref_length - 1.0) < 1e-6
        assert abs(fc.cl) < 1e-3 and abs(fc.cm) < 1e-3
        assert abs(fc.cd - cd_ref) / cd_ref < 0.05
        assert fc.cdp > 0 and fc.cdf > 0


@pytest.mark.slow
def test_farfield_outflow_equals_dirichlet(oracle_mod):
    """tests/test_postproc.py:87-118: r=100, 101x151, Re=20: omega-only
    outflow leaves Cd unchanged to 1e-6 and keeps the symmetry."""
    cd = {}
    for bc in ("dirichlet", "outflow"):
        fc = steady(oracle_mod, 101, 151, 20.0, outer=100.0, farfield_bc=bc).force_coeffs()
        assert abs(fc.cl) < 1e-3
        cd[bc] = fc.cd
    assert abs(cd["outflow"] - cd["dirichlet"]) < 1e-6


@pytest.mark.slow
def test_angle_of_attack_far_field(oracle_mod):
    """tests/test_postproc.py:121-142: far-field psi = cos(a) y - sin(a) x."""
    for adeg in (0.0, 12.0):
        s = steady(oracle_mod, 121, 121, 20.0, alpha_deg=adeg)
        ff = slice(s.imax * (s.jmax - 1), s.imax * s.jmax)
        target = s.ca * s.yphys[ff] - s.sa * s.xphys[ff]
        assert np.max(np.abs(s.psi[ff] - target)) < 1e-9


@pytest.mark.slow
def test_documented_drag_181(oracle_mod):
    """docs/verification.rst:132-147: steady Cd on the 181x181 analytic grid,
    Re=20: 2.036, Re=40: 1.522 (three significant digits as documented)."""
    for re, cd_doc in [(20.0, 2.036), (40.0, 1.522)]:
        fc = steady(oracle_mod, 181, 181, re).force_coeffs()
        assert abs(fc.cd - cd_doc) < 1.5e-3, (re, fc.cd)


def test_unsteady_bdf2_history(oracle_mod):
    """BDF2 from a cold start with zero history, solving at t_start first
    (vorti2d/solver.py:104-107,176-191)."""
    xg, yg = oracle_mod.generate_cylinder(25, 17)
    s = oracle_mod.OracleSolver(xg, yg, re=40.0, dt_phys=0.5, t_end=1.0, rot_speed=0.5,
                                rot_until=2.0, pseudo_tol=1e-9, max_pseudo_iter=50)
    assert s.times() == [0.0, 0.5, 1.0]
    s.advance(0.0)
    assert np.array_equal(s.omeold, s.ome)
    assert not np.any(s.omeoldold)
    prev = s.ome.copy()
    s.advance(0.5)
    assert np.array_equal(s.omeoldold, prev)
