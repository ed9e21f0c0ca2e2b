"""Batched steady sweeps: instances solved concurrently on one GPU (one
handle and stream each, driven from a thread pool) give the same answers as
the same instances solved one after another."""
import math

import numpy as np
import pytest


def _small_cases(v2d):
    from vorti2d_b200.batch import Case
    # plain Newton from the free stream converges on these (checked against
    # the oracle's direct-solve Newton): cylinders 65x49 up to Re 80, the
    # 65x33 NACA-0012 section at Re 5
    cyl = v2d.generate_cylinder(65, 49)
    naca = v2d.generate_naca0012(65, 33)
    cases = []
    for k, (re, a) in enumerate([(40.0, 0.0), (60.0, 4.0), (30.0, -6.0), (80.0, 2.0)]):
        cases.append(Case(f"cyl_{k}", *cyl, re, a))
    for k, (re, a) in enumerate([(5.0, 2.0), (5.0, -3.0)]):
        cases.append(Case(f"naca_{k}", *naca, re, a, 1.0))
    return cases


def test_sweep_cases_are_seeded():
    from vorti2d_b200.batch import sweep_cases
    a, b = sweep_cases(seed=3, n_each=2), sweep_cases(seed=3, n_each=2)
    assert [(c.name, c.re, c.alpha_deg) for c in a] == [(c.name, c.re, c.alpha_deg) for c in b]
    assert len(a) == 6
    for c in a:
        assert 50.0 <= c.re <= 1000.0 and -8.0 <= c.alpha_deg <= 8.0
    shapes = sorted({c.xg.shape for c in a})
    assert shapes == [(129, 129), (181, 181), (257, 129)]


@pytest.mark.gpu
def test_concurrent_equals_sequential(v2d):
    from vorti2d_b200.batch import run_sweep
    cases = _small_cases(v2d)
    seq = run_sweep(cases, workers=1, precision="fp64", pseudo_tol=1e-11)
    par = run_sweep(cases, workers=6, precision="fp64", pseudo_tol=1e-11)
    assert seq.converged == len(cases), [(r.name, r.newton_iters, r.res, r.error)
                                         for r in seq.results]
    assert par.converged == len(cases), [(r.name, r.newton_iters, r.res, r.error)
                                         for r in par.results]
    for a, b in zip(seq.results, par.results):
        assert a.name == b.name and a.newton_iters == b.newton_iters, (a, b)
        for key in ("cd", "cl", "cm"):
            x, y = getattr(a, key), getattr(b, key)
            assert math.isfinite(x) and abs(x - y) <= 1e-10 * max(1.0, abs(x)), (a.name, key, x, y)
    assert seq.newton_iters == par.newton_iters > 0


@pytest.mark.gpu
def test_sweep_matches_oracle_forces(v2d, oracle_mod):
    """Converged concurrent instances reproduce the oracle's steady forces."""
    from vorti2d_b200.batch import run_sweep
    cases = [c for c in _small_cases(v2d) if c.name in ("cyl_1", "naca_0")]
    par = run_sweep(cases, workers=2, precision="mixed", pseudo_tol=1e-11)
    for c, r in zip(cases, par.results):
        assert r.converged, r
        o = oracle_mod.OracleSolver(c.xg, c.yg, re=c.re, alpha_deg=c.alpha_deg, steady=True,
                                    pseudo_tol=1e-11, max_pseudo_iter=30)
        o.advance(0.0)
        fc = oracle_mod.compute_force_coeffs(o.imax, o.jmax, o.re, o.dksi, o.deta, o.beta,
                                             o.gama, o.detadx, o.detady, o.xphys, o.yphys,
                                             o.ome, ref_length=c.ref_length)
        for key in ("cd", "cl"):
            want = getattr(fc, key)
            assert abs(getattr(r, key) - want) <= 1e-8 * max(1.0, abs(want)), (c.name, key)


@pytest.mark.gpu
def test_reynolds_continuation_reaches_the_oracle_state(v2d, oracle_mod):
    """A sweep instance solved along Re 80 -> 120 -> 150 (set_re on one
    handle, each Reynolds number from the previous state) ends on the steady
    state the oracle's plain Newton finds at Re 150 (65x49 cylinder, alpha
    0, where plain Newton converges too)."""
    from vorti2d_b200.batch import Case, run_sweep
    xg, yg = v2d.generate_cylinder(65, 49)
    case = Case("cyl_cont", xg, yg, 150.0, 0.0)
    out = run_sweep([case], workers=1, precision="fp64", pseudo_tol=1e-11, continuation=1.5,
                    re_start=80.0)
    r = out.results[0]
    assert r.converged and r.rungs == 3 and r.re_reached == 150.0, r
    o = oracle_mod.OracleSolver(xg, yg, re=150.0, alpha_deg=0.0, steady=True, pseudo_tol=1e-11,
                                max_pseudo_iter=30)
    o.advance(0.0)
    fc = oracle_mod.compute_force_coeffs(o.imax, o.jmax, o.re, o.dksi, o.deta, o.beta, o.gama,
                                         o.detadx, o.detady, o.xphys, o.yphys, o.ome)
    assert abs(r.cd - fc.cd) <= 1e-8 * max(1.0, abs(fc.cd)), (r.cd, fc.cd)
    assert abs(r.cl - fc.cl) <= 1e-8, (r.cl, fc.cl)
