"""GPU parity of the kernel seam against the CPU restatement (oracle).

Metrics, COO triplets, right-hand sides and the canonical CSR are compared
bit for bit: the kernels evaluate the reference's expressions in the same
order without FMA contraction, as the oracle does.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from cases import local_layout, smooth_state, to_local

pytestmark = pytest.mark.gpu

SIZES = [(5, 4), (9, 7), (25, 17), (33, 21), (64, 48), (129, 129)]


@pytest.mark.parametrize("imax,jmax", SIZES)
def test_metrics_bit_exact(v2d, oracle_mod, imax, jmax):
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    dk, de = 1.0 / (imax - 1), 1.0 / (jmax - 1)
    got = v2d.core.compute_metrics(dk, de, xg, yg)
    ref = oracle_mod.core().compute_metrics(dk, de, xg, yg)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)


def test_metrics_naca_bit_exact(v2d, oracle_mod):
    xg, yg = v2d.generate_naca0012(65, 33)
    got = v2d.core.compute_metrics(1 / 64, 1 / 32, xg, yg)
    ref = oracle_mod.core().compute_metrics(1 / 64, 1 / 32, xg, yg)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)


CASES = [
    # re, invdtau, inv2dt, urot, ff_bc, alpha_deg
    (40.0, 0.0, 0.0, 0.0, 0, 0.0),
    (80.0, 0.0, 1.0 / 0.4, 0.3, 1, 0.0),
    (100.0, 0.5, 2.5, -0.2, 2, 12.0),
    (500.0, 1.0, 0.0, 0.0, 1, -8.0),
]


@pytest.mark.parametrize("imax,jmax", [(5, 4), (25, 17), (64, 48)])
@pytest.mark.parametrize("case", CASES)
def test_assemble_coo_bit_exact(v2d, oracle_mod, imax, jmax, case):
    re, invdtau, inv2dt, urot, ff_bc, adeg = case
    ca, sa = np.cos(np.radians(adeg)), np.sin(np.radians(adeg))
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    dk, de = 1.0 / (imax - 1), 1.0 / (jmax - 1)
    M = oracle_mod.core().compute_metrics(dk, de, xg, yg)
    st = smooth_state(M[8], M[9])
    N = imax * jmax
    for r0, r1 in [(0, 2 * N), (0, N), (N, 2 * N), (N // 3, N + N // 2)]:
        maxnnz = (r1 - r0) * 13
        args = (imax, jmax, re, invdtau, inv2dt, urot, dk, de, *M, *st, r0, r1, maxnnz,
                ff_bc, ca, sa)
        gi, gj, gv, gn, gb = v2d.core.assemble_coo(*args)
        oi, oj, ov, on, ob = oracle_mod.core().assemble_coo(*args)
        assert gn == on
        assert np.array_equal(gi[:gn], oi[:on])
        assert np.array_equal(gj[:gn], oj[:on])
        assert np.array_equal(gv[:gn], ov[:on])
        assert np.array_equal(gb, ob)


def test_assemble_coo_nnz_formula(v2d, oracle_mod):
    """nnz(ff_bc=0) = 23*imax*(jmax-2) + 7*imax (ψ interior 10, ω interior 13,
    wall ψ 1 + ω 4, far field 1 + 1)."""
    imax, jmax = 33, 21
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / 32, 1 / 20, xg, yg)
    N = imax * jmax
    z = np.zeros(N)
    *_, nnz, _ = v2d.core.assemble_coo(imax, jmax, 40.0, 0, 0, 0, 1 / 32, 1 / 20, *M, z, z, z, z,
                                       0, 2 * N, 26 * N, 0, 1.0, 0.0)
    assert nnz == 23 * imax * (jmax - 2) + 7 * imax


def test_assemble_coo_capacity_error(v2d, oracle_mod):
    imax, jmax = 9, 7
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / 8, 1 / 6, xg, yg)
    z = np.zeros(imax * jmax)
    with pytest.raises(Exception):
        v2d.core.assemble_coo(imax, jmax, 40.0, 0, 0, 0, 1 / 8, 1 / 6, *M, z, z, z, z, 0,
                              2 * imax * jmax, 10, 0, 1.0, 0.0)


@pytest.mark.parametrize("imax,jmax", [(25, 17), (33, 21)])
def test_local_metrics_and_assembly_bit_exact(v2d, oracle_mod, imax, jmax):
    ni, gxs, gxm, il0, il1, gc, lg = local_layout(imax, jmax)
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    xgl = xg[:ni][gc]
    ygl = yg[:ni][gc]
    dk, de = 1.0 / (imax - 1), 1.0 / (jmax - 1)
    got = v2d.core.compute_metrics_local(il0, il1, dk, de, xgl, ygl)
    ref = oracle_mod.core().compute_metrics_local(il0, il1, dk, de, xgl, ygl)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
    M = oracle_mod.core().compute_metrics(dk, de, xg, yg)
    st = smooth_state(M[8], M[9])
    loc = [to_local(f, imax, jmax, gxm, gc) for f in (*M, *st)]
    nloc = 2 * ni * jmax
    args = (gxm, jmax, il0, il1, 80.0, 0.0, 2.5, 0.3, dk, de, *loc, 0, nloc, lg, 14 * nloc, 1,
            1.0, 0.0)
    gi, gj, gv, gn, gb = v2d.core.assemble_coo_local(*args)
    oi, oj, ov, on, ob = oracle_mod.core().assemble_coo_local(*args)
    assert gn == on
    assert np.array_equal(gi[:gn], oi[:on]) and np.array_equal(gj[:gn], oj[:on])
    assert np.array_equal(gv[:gn], ov[:on]) and np.array_equal(gb, ob)


def test_node_neighbors(v2d, oracle_mod):
    for imax in (4, 9, 181):
        for i in (1, 2, imax - 1, imax):
            for j in (2, 5):
                assert v2d.core.node_neighbors(i, j, imax) == oracle_mod.core().node_neighbors(i, j, imax)


@pytest.mark.parametrize("ff_bc,adeg", [(0, 0.0), (1, 0.0), (2, 8.0)])
def test_solver_csr_bit_exact(v2d, oracle_mod, ff_bc, adeg):
    """Device Newton system == scipy canonical CSR of the oracle's COO
    (vorti2d/petsc_solver.py:80-89): indptr/indices/data/b bit for bit."""
    imax, jmax = 33, 25
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    bc = {0: "dirichlet", 1: "outflow", 2: "outflow_psi"}[ff_bc]
    cfg = v2d.Config(re=100.0, steady=False, dt_phys=0.2, farfield_bc=bc, alpha_deg=adeg,
                     verbose=False)
    s = v2d.Solver(cfg, mesh=(xg, yg))
    M = oracle_mod.core().compute_metrics(1 / 32, 1 / 24, xg, yg)
    st = smooth_state(M[8], M[9])
    s.set_state(*st)
    ip, ix, dv, b = s.dev.system(urot=0.4)
    N = imax * jmax
    ci, cj, cv, nnz, ob = oracle_mod.core().assemble_coo(
        imax, jmax, 100.0, 0.0, 2.5, 0.4, 1 / 32, 1 / 24, *M, *st, 0, 2 * N, 26 * N, ff_bc,
        cfg.cos_alpha(), cfg.sin_alpha())
    A = sp.csr_matrix((cv[:nnz], (ci[:nnz].astype(np.int64), cj[:nnz].astype(np.int64))),
                      shape=(2 * N, 2 * N))
    assert A.has_canonical_format
    assert np.array_equal(ip, A.indptr)
    assert np.array_equal(ix, A.indices)
    assert np.array_equal(dv, A.data)
    assert np.array_equal(b, ob)
    s.close()


def test_forces_vs_oracle(v2d, oracle_mod):
    imax, jmax = 65, 49
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / 64, 1 / 48, xg, yg)
    _, ome, _, _ = smooth_state(M[8], M[9])
    for ref_length, mref in [(None, (0.0, 0.0)), (1.0, (0.25, -0.1))]:
        args = (imax, jmax, 40.0, 1 / 64, 1 / 48, M[2], M[3], M[6], M[7], M[8], M[9], ome)
        g = v2d.compute_force_coeffs(*args, ref_length=ref_length, moment_ref=mref)
        o = oracle_mod.compute_force_coeffs(*args, ref_length=ref_length, moment_ref=mref)
        for k in ("cd", "cl", "cm", "cdp", "cdf", "clp", "clf", "cmp", "cmf", "ref_length"):
            a, bb = getattr(g, k), getattr(o, k)
            assert abs(a - bb) <= 1e-12 * max(1.0, abs(bb)), (k, a, bb)


def test_linsys_seam_canonical_csr_and_solve(v2d, oracle_mod):
    """MumpsSolver seam: COO (shuffled, with duplicates) -> canonical CSR equal
    to scipy's, and the GMRES solution of a diagonally dominant system."""
    rng = np.random.default_rng(0)
    n = 400
    rows, cols, vals = [], [], []
    for r in range(n):
        for c in {r, (r + 1) % n, (r - 1) % n, (r + 17) % n}:
            rows.append(r); cols.append(c); vals.append(4.0 if c == r else rng.uniform(-1, 1))
    rows += [5, 5, 7]; cols += [5, 6, 7]; vals += [0.5, 0.25, 1.0]   # duplicates
    perm = rng.permutation(len(rows))
    ci = np.array(rows)[perm]; cj = np.array(cols)[perm]; cv = np.array(vals)[perm]
    b = rng.standard_normal(n)
    lin = v2d.MumpsSolver(n, block_layout=2, restart=30, rtol=1e-12, precond="bjacobi")
    lin.assemble(ci, cj, cv, b)
    A = sp.csr_matrix((cv, (ci, cj)), shape=(n, n))
    ip, ix, dv = lin.csr()
    assert np.array_equal(ip, A.indptr) and np.array_equal(ix, A.indices)
    assert np.allclose(dv, A.data, rtol=1e-15, atol=0)
    x = lin.solve()
    assert np.linalg.norm(A @ x - b) <= 1e-11 * np.linalg.norm(b)
    # value refresh keeps the pattern
    lin.assemble(ci, cj, 2.0 * cv, b)
    x2 = lin.solve()
    assert np.allclose(x2, 0.5 * x, rtol=1e-8, atol=1e-12)
    with pytest.raises(ValueError):
        lin.assemble(cj, ci, cv, b)    # different pattern
    lin.destroy()


def test_state_round_trip_through_pinned_buffers(v2d, oracle_mod):
    """Solver.set_state -> get_state(out=...) into pinned host buffers returns
    the arrays bit for bit, matches get_state(), and rejects bad buffers."""
    import torch
    imax, jmax = 33, 25
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    cfg = v2d.Config(re=100.0, steady=False, dt_phys=0.2, verbose=False)
    s = v2d.Solver(cfg, mesh=(xg, yg))
    N = imax * jmax
    rng = np.random.default_rng(7)
    st = [rng.standard_normal(N) for _ in range(4)]
    s.set_state(*st)
    host = [torch.empty(N, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
    got = s.get_state(out=host)
    assert all(g is h for g, h in zip(got, host))
    for h, a, b in zip(host, st, s.get_state()):
        assert np.array_equal(h, a)
        assert np.array_equal(b, a)
    assert np.array_equal(s.psi, st[0]) and np.array_equal(s.omeoldold, st[3])
    with pytest.raises(ValueError):
        s.get_state(out=host[:3])
    with pytest.raises(ValueError):
        s.get_state(out=[np.zeros(N, dtype=np.float32)] + host[1:])
    with pytest.raises(ValueError):
        s.get_state(out=[np.zeros(N + 1)] + host[1:])
    with pytest.raises(ValueError):
        s.get_state(out=[np.zeros((N, 2))[:, 0]] + host[1:])
    s.close()


def test_set_state_keeps_factors_when_reused_across_steps(v2d, oracle_mod):
    """With LU factors kept across steps, copying the state out and back in
    between steps (set_state) changes nothing: the next step equals that of
    a twin solver that kept its state on the device, and no extra
    factorization is needed for it."""
    xg, yg = oracle_mod.generate_cylinder(65, 49)
    kw = dict(re=100.0, steady=False, dt_phys=0.2, rot_speed=0.5, rot_until=2.0,
              farfield_bc="outflow", verbose=False, precision="mixed", precond="lu",
              lu_reuse_its=12, lu_reuse_steps=True, max_pseudo_iter=5)
    a = v2d.Solver(v2d.Config(**kw), mesh=(xg, yg))
    b = v2d.Solver(v2d.Config(**kw), mesh=(xg, yg))
    times = a.times()
    for t in times[:3]:
        a.advance(t)
        b.advance(t)
    b.set_state(*b.get_state())
    a.advance(times[3])
    b.advance(times[3])
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.max(np.abs(x - y)) <= 1e-12 * max(1.0, np.max(np.abs(x)))
    assert a.newton_log[-1][1:3] == b.newton_log[-1][1:3]
    a.close()
    b.close()
