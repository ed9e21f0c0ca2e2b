"""The linear-solver seam as the reference drives it: the replicated Newton
loop of vorti2d/solver.py:117-145 -- assemble_coo for the owned rows,
MumpsSolver.assemble, MumpsSolver.solve, q += dq, res = ||dq|| / (2N) -- run
with vorti2d_b200's core and MumpsSolver, against the oracle's steady solve
(SuperLU standing in for the reference's MUMPS).  The seam's default
preconditioner is the multifrontal LU, with the O-grid shape recognised from
the pattern."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    return np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b)))


def reference_loop(core, lin, imax, jmax, re, xg, yg, ff_bc=0, alpha_deg=0.0, tol=1e-12,
                   max_it=40):
    """vorti2d/solver.py:103-145 written against the seam objects only."""
    dk, de = 1.0 / (imax - 1), 1.0 / (jmax - 1)
    M = core.compute_metrics(dk, de, xg, yg)
    N = imax * jmax
    ca, sa = np.cos(np.radians(alpha_deg)), np.sin(np.radians(alpha_deg))
    psi, ome = np.zeros(N), np.zeros(N)
    ff = slice(imax * (jmax - 1), N)
    psi[ff] = ca * M[9][ff] - sa * M[8][ff]
    r0, r1 = lin.row_range()
    maxnnz = (r1 - r0) * 13
    res, it = 1.0e5, 0
    while res > tol and it < max_it:
        ci, cj, cv, nnz, b = core.assemble_coo(imax, jmax, re, 0.0, 0.0, 0.0, dk, de, *M, psi,
                                               ome, ome, ome, r0, r1, maxnnz, ff_bc, ca, sa)
        lin.assemble(ci[:nnz], cj[:nnz], cv[:nnz], b)
        dq = lin.solve()
        psi += dq[:N]
        ome += dq[N:]
        res = float(np.linalg.norm(dq) / (2.0 * N))
        it += 1
    return psi, ome, res, it, M


def test_steady_129_through_the_seam_matches_oracle(v2d, oracle_mod):
    """Config 1 (129x129 cylinder, Re 40, Dirichlet far field, pure Newton to
    ||dq||/(2N) < 1e-12): psi/omega within 1e-9 and Cl/Cd/Cm within 1e-8 of the
    oracle, each solve refactoring the Jacobian like MUMPS."""
    imax = jmax = 129
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    lin = v2d.MumpsSolver(2 * imax * jmax)
    assert lin.row_range() == (0, 2 * imax * jmax)
    psi, ome, res, it, M = reference_loop(v2d.core, lin, imax, jmax, 40.0, xg, yg)
    ref = oracle_mod.OracleSolver(xg, yg, re=40.0, steady=True, pseudo_tol=1e-12,
                                  max_pseudo_iter=40).run()
    assert res <= 1e-12 and abs(it - ref.history[-1][1]) <= 1
    assert _close(psi, ref.psi, 1e-9) and _close(ome, ref.ome, 1e-9)
    args = (imax, jmax, 40.0, 1 / 128, 1 / 128, M[2], M[3], M[6], M[7], M[8], M[9])
    fg = oracle_mod.compute_force_coeffs(*args, ome)
    fo = ref.force_coeffs()
    for k in ("cd", "cl", "cm"):
        assert abs(getattr(fg, k) - getattr(fo, k)) <= 1e-8, k
    st = lin.last_stats
    assert st.converged and st.iterations <= 3      # a direct solve refined by GMRES
    t = lin.timings()
    assert set(t) == {"csr_assemble", "linsolve", "gather_toall", "n_solves"}
    assert t["n_solves"] == it
    lin.destroy()


# shapes on which the reference's steady Newton converges from the free stream
# (on coarser ones, e.g. 33x21 or 24x13, it does not: the oracle stalls there
# too)
@pytest.mark.parametrize("imax,jmax,ff_bc,alpha", [(33, 25, 1, 4.0), (64, 48, 2, -8.0),
                                                   (65, 49, 0, 4.0)])
@pytest.mark.parametrize("grid", [False, True])
def test_seam_lu_shapes_and_far_field_bcs(v2d, oracle_mod, imax, jmax, ff_bc, alpha, grid):
    """The grid recognised from the pattern (or given) on odd/even shapes and
    every far-field BC; a steady solve at Re 20 equals the oracle's."""
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    lin = v2d.MumpsSolver(2 * imax * jmax, grid=(imax, jmax) if grid else None)
    psi, ome, res, it, _ = reference_loop(v2d.core, lin, imax, jmax, 20.0, xg, yg, ff_bc, alpha)
    bc = {0: "dirichlet", 1: "outflow", 2: "outflow_psi"}[ff_bc]
    ref = oracle_mod.OracleSolver(xg, yg, re=20.0, steady=True, pseudo_tol=1e-12,
                                  max_pseudo_iter=40, farfield_bc=bc, alpha_deg=alpha).run()
    assert res <= 1e-12
    assert _close(psi, ref.psi, 1e-9) and _close(ome, ref.ome, 1e-9)
    lin.destroy()


def test_seam_lu_rejects_systems_without_grid(v2d):
    """A matrix that is not an O-grid psi-omega system cannot be ordered for
    the LU without its shape: assemble raises with the reason, and a wrong
    explicit shape is refused up front."""
    n = 2 * 11 * 13
    lin = v2d.MumpsSolver(n)
    idx = np.arange(n)
    with pytest.raises(ValueError, match="O-grid"):
        lin.assemble(idx, idx, np.full(n, 2.0), np.ones(n))
    lin.destroy()
    with pytest.raises(ValueError):
        v2d.MumpsSolver(n, grid=(12, 13))
