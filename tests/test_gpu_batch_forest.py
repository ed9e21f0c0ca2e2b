"""The batched steady solve (v2d_batch_*): uneven instances advanced by Newton
together as the diagonal blocks of one block-diagonal system (one assembly
launch, one factorization over the forest of separator trees, one GMRES, one
update launch per iteration).  Each instance must end where its own
single-instance solve ends (fields within 1e-9, forces within 1e-8), and on
the oracle's steady forces; a frozen instance must not move."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(v2d, oracle_mod):
    from vorti2d_b200.batch import Case
    cyl33 = oracle_mod.generate_cylinder(33, 25)
    cyl65 = oracle_mod.generate_cylinder(65, 49)
    naca = v2d.generate_naca0012(65, 33)
    return [Case("cyl33_a", *cyl33, 20.0, 0.0), Case("cyl65_a", *cyl65, 40.0, 4.0),
            Case("naca65_a", *naca, 5.0, 3.0, 1.0), Case("cyl33_b", *cyl33, 30.0, -6.0),
            Case("cyl65_b", *cyl65, 25.0, 8.0)]


def _single(v2d, c, precision):
    from vorti2d_b200.batch import _config
    cfg = _config(c, precision, 30, 1e-12, 300)
    s = v2d.Solver(cfg, mesh=(c.xg, c.yg))
    s.advance(0.0)
    out = (s.get_state()[:2], s.force_coeffs(), s.newton_log[-1][1])
    s.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_instance_solves(v2d, oracle_mod, precision):
    from vorti2d_b200.batch import run_sweep_batched
    cases = _cases(v2d, oracle_mod)
    res = run_sweep_batched(cases, precision=precision, max_newton=30, pseudo_tol=1e-12)
    assert res.converged == len(cases), [(r.name, r.res, r.error) for r in res.results]
    for c, r in zip(cases, res.results):
        (psi, ome), fc, its = _single(v2d, c, precision)
        assert abs(r.newton_iters - its) <= 1, (c.name, r.newton_iters, its)
        for k in ("cd", "cl", "cm"):
            assert abs(getattr(r, k) - getattr(fc, k)) <= 1e-8, (c.name, k)
    # the oracle's steady forces on two instances
    for c, r in ((cases[1], res.results[1]), (cases[2], res.results[2])):
        o = oracle_mod.OracleSolver(c.xg, c.yg, re=c.re, alpha_deg=c.alpha_deg, steady=True,
                                    pseudo_tol=1e-12, max_pseudo_iter=40).run()
        fo = oracle_mod.compute_force_coeffs(o.imax, o.jmax, o.re, o.dksi, o.deta, o.beta,
                                             o.gama, o.detadx, o.detady, o.xphys, o.yphys,
                                             o.ome, ref_length=c.ref_length)
        for k in ("cd", "cl", "cm"):
            assert abs(getattr(r, k) - getattr(fo, k)) <= 1e-8, (c.name, k)


def test_batch_fields_and_frozen_instance(v2d, oracle_mod):
    """Fields of the batched solve equal the single-instance fields to 1e-9;
    an instance frozen from the start keeps its initial state."""
    from vorti2d_b200 import _lib
    from vorti2d_b200.batch import _config
    from vorti2d_b200.solver import solver_params
    cases = _cases(v2d, oracle_mod)[:3]
    n = len(cases)
    cfgs = [_config(c, "fp64", 30, 1e-12, 300) for c in cases]
    params = (_lib.SolverParams * n)(*[solver_params(c) for c in cfgs])
    xs = [np.asfortranarray(c.xg) for c in cases]
    ys = [np.asfortranarray(c.yg) for c in cases]
    imax = np.array([x.shape[0] for x in xs], dtype=np.intc)
    jmax = np.array([x.shape[1] for x in xs], dtype=np.intc)
    h = ctypes.c_void_p()
    _lib.check(_lib.lib().v2d_batch_create(n, _lib.iptr(imax), _lib.iptr(jmax),
                                            (_lib._dp * n)(*[_lib.dptr(x) for x in xs]),
                                            (_lib._dp * n)(*[_lib.dptr(y) for y in ys]), params,
                                            ctypes.byref(h)))

    def state(i):
        s = ctypes.c_void_p()
        _lib.check(_lib.lib().v2d_batch_instance(h, i, ctypes.byref(s)))
        N = int(imax[i] * jmax[i])
        a, b = np.zeros(N), np.zeros(N)
        _lib.check(_lib.lib().v2d_solver_get_state(s, _lib.dptr(a), _lib.dptr(b), None, None))
        return a, b

    psi2, ome2 = state(2)
    active = np.array([1, 1, 0], dtype=np.intc)
    _lib.check(_lib.lib().v2d_batch_set_active(h, _lib.iptr(active)))
    res = np.zeros(n)
    for _ in range(30):
        st = _lib.LinStats()
        _lib.check(_lib.lib().v2d_batch_newton(h, _lib.dptr(res), None, ctypes.byref(st)))
        assert res[2] == 0.0
        if max(res[:2]) <= 1e-12:
            break
    assert max(res[:2]) <= 1e-12
    for i in range(2):
        (psi, ome), _, _ = _single(v2d, cases[i], "fp64")
        a, b = state(i)
        assert np.max(np.abs(a - psi)) <= 1e-9 * max(1.0, np.abs(psi).max())
        assert np.max(np.abs(b - ome)) <= 1e-9 * max(1.0, np.abs(ome).max())
    a, b = state(2)
    assert np.array_equal(a, psi2) and np.array_equal(b, ome2)
    _lib.lib().v2d_batch_destroy(h)


def test_sweep_96_converges_where_the_oracle_does(v2d):
    """The 96-instance sweep (seed 0) batched on the device with the bench's
    rules (FP64, at most 20 Newton iterations, GMRES capped at 30 per Newton
    step, frozen past 1000x the first update norm) converges on exactly the
    instances the oracle's pure-Newton solves converge on
    (tests/golden/sweep_oracle_96.json, tests/golden/make_sweep_oracle.py),
    with the same forces there (1e-8)."""
    import json
    import os
    from vorti2d_b200.batch import run_sweep_batched, sweep_cases
    with open(os.path.join(os.path.dirname(__file__), "golden", "sweep_oracle_96.json")) as fh:
        ref = {r["name"]: r for r in json.load(fh)["cases"]}
    res = run_sweep_batched(sweep_cases(seed=0), precision="fp64", krylov_max_it=30)
    got = {r.name: r for r in res.results}
    assert set(got) == set(ref)
    conv = sorted(n for n, r in got.items() if r.converged)
    assert conv == sorted(n for n, r in ref.items() if r["converged"]), conv
    for n in conv:
        for k in ("cd", "cl", "cm"):
            assert abs(getattr(got[n], k) - ref[n][k]) <= 1e-8, (n, k, getattr(got[n], k), ref[n][k])
