"""The LU preconditioner solve in its two launch forms: one dataflow launch
over the whole front tree (the default, Config.lu_solve = "flow") and one
launch per level and sweep ("levels").  Both run the same work items with the
same arithmetic, and each output entry is written by exactly one item, so
the Newton updates agree bit for bit."""
import ctypes

import numpy as np
import pytest

from cases import smooth_state

pytestmark = pytest.mark.gpu

SHAPES = [(9, 7, 1), (33, 21, 1), (64, 48, 0), (129, 65, 2), (181, 181, 1)]


def _solver(v2d, xg, yg, bc, precision, lu_solve, item_rows=None):
    cfg = v2d.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                     re=80.0, steady=False, dt_phys=0.2, farfield_bc=bc, alpha_deg=4.0,
                     precision=precision, precond="lu", ksp_rtol=1e-12, lu_solve=lu_solve,
                     lu_item_rows=item_rows)
    return v2d.Solver(cfg, mesh=(xg, yg))


@pytest.mark.parametrize("imax,jmax,ff_bc", SHAPES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_flow_newton_update_equals_levels(v2d, oracle_mod, imax, jmax, ff_bc, precision):
    bc = {0: "dirichlet", 1: "outflow", 2: "outflow_psi"}[ff_bc]
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / (imax - 1), 1 / (jmax - 1), xg, yg)
    st = smooth_state(M[8], M[9])
    out = []
    for form in ("levels", "flow"):
        s = _solver(v2d, xg, yg, bc, precision, form)
        s.set_state(*st)
        code, res, lin = s.dev.newton(0.3)
        assert code == 0, v2d._lib.last_error()
        out.append((np.concatenate(s.dev.get_state()[:2]), lin.iterations, res))
        s.close()
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][2] == out[1][2]


def test_launch_lists_181(v2d, oracle_mod):
    """181x181: the dataflow solve is a single launch, the level form 22 (11
    levels, forward and backward); the device time of both is printed."""
    from vorti2d_b200 import _lib
    xg, yg = oracle_mod.generate_cylinder(181, 181)
    M = oracle_mod.core().compute_metrics(1 / 180, 1 / 180, xg, yg)
    st = smooth_state(M[8], M[9])
    totals = {}
    for form in ("levels", "flow"):
        s = _solver(v2d, xg, yg, "outflow", "mixed", form)
        s.set_state(*st)
        code, _, _ = s.dev.newton(0.3)
        assert code == 0, v2d._lib.last_error()
        cap = 64
        ms = (ctypes.c_double * cap)()
        codes = (ctypes.c_int * cap)()
        n = ctypes.c_int()
        _lib.check(_lib.lib().v2d_solver_time_lu_launches(s.dev.h, 5, 0, ms, codes, cap,
                                                         ctypes.byref(n)))
        kinds = [codes[k] // 1000 for k in range(n.value)]
        if form == "flow":
            assert kinds == [2], kinds
        else:
            assert kinds == [0] * 11 + [1] * 11, kinds
        totals[form] = sum(ms[k] for k in range(n.value))
        s.close()
    print(f"LU solve 181x181 mixed, warm: levels {totals['levels']:.3f} ms, "
          f"dataflow {totals['flow']:.3f} ms")


def test_tuned_item_split_gives_the_same_newton_update(v2d, oracle_mod, tmp_path):
    """The autotuner's split (vorti2d_b200.tune) is recorded to a file, read
    back into a fresh solver, and the Newton update with it equals the
    default split's to 1e-10 relative (the same products, partial sums in a
    split-dependent order, each solve to its tolerance)."""
    from vorti2d_b200 import tune
    xg, yg = oracle_mod.generate_cylinder(65, 49)
    M = oracle_mod.core().compute_metrics(1 / 64, 1 / 48, xg, yg)
    st = smooth_state(M[8], M[9])
    path = str(tmp_path / "lu_tuning.json")

    def update(s):
        s.set_state(*st)
        code, _, _ = s.dev.newton(0.3)
        assert code == 0, v2d._lib.last_error()
        return np.concatenate(s.dev.get_state()[:2]) - np.concatenate(st[:2])

    s = _solver(v2d, xg, yg, "outflow", "mixed", "flow")
    default = update(s)
    rec = tune.tune_lu_solve(s, sweeps=1, reps=5, path=path)
    assert len(rec["rows"]) == len(tune.item_rows(s)) and rec["ms"] <= rec["default_ms"]
    s.close()
    s = _solver(v2d, xg, yg, "outflow", "mixed", "flow")
    assert tune.load_tuning(s, path) and tune.item_rows(s) == rec["rows"]
    tuned = update(s)
    s.close()
    assert np.max(np.abs(default - tuned)) <= 1e-10 * np.abs(default).max()


@pytest.mark.parametrize("imax,jmax,ff_bc", [(33, 21, 1), (129, 65, 2), (181, 181, 1)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gathered_split(v2d, oracle_mod, imax, jmax, ff_bc, precision):
    """Negative rows-per-item entries (gather items first, then rows that
    read the gathered vectors): the dataflow and per-level forms agree bit
    for bit, and the Newton update equals the one of the plain split of the
    same row counts to 1e-10 relative (the same products; only where the
    right-hand side is gathered changes)."""
    from vorti2d_b200 import tune
    bc = {0: "dirichlet", 1: "outflow", 2: "outflow_psi"}[ff_bc]
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / (imax - 1), 1 / (jmax - 1), xg, yg)
    st = smooth_state(M[8], M[9])
    probe = _solver(v2d, xg, yg, bc, precision, "flow")
    nl = len(tune.item_rows(probe))
    probe.close()
    plain = [0 if L < 2 else (16 if L % 2 else 8) for L in range(nl)]
    gathered = [0 if L < 2 else -r for L, r in enumerate(plain)]
    out = {}
    for name, rows, form in (("plain", plain, "flow"), ("gathered", gathered, "flow"),
                             ("gathered_levels", gathered, "levels")):
        s = _solver(v2d, xg, yg, bc, precision, form, item_rows=rows)
        assert tune.item_rows(s) == rows
        s.set_state(*st)
        code, res, lin = s.dev.newton(0.3)
        assert code == 0, v2d._lib.last_error()
        out[name] = np.concatenate(s.dev.get_state()[:2]) - np.concatenate(st[:2])
        s.close()
    assert np.array_equal(out["gathered"], out["gathered_levels"])
    scale = np.abs(out["plain"]).max()
    assert np.max(np.abs(out["plain"] - out["gathered"])) <= 1e-10 * scale


@pytest.mark.parametrize("imax,jmax,ff_bc", [(33, 21, 1), (129, 65, 2), (181, 181, 1)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_split_launches(v2d, oracle_mod, imax, jmax, ff_bc, precision):
    """The split form (tree levels [0, L) as launches of their own, forward
    before and backward after the upper levels' launch, in 128-thread CTAs)
    gives the Newton update of the one-launch form to 1e-10 relative, for
    every split level the tuner may pick."""
    from vorti2d_b200 import tune
    bc = {0: "dirichlet", 1: "outflow", 2: "outflow_psi"}[ff_bc]
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / (imax - 1), 1 / (jmax - 1), xg, yg)
    st = smooth_state(M[8], M[9])

    def update(split):
        s = _solver(v2d, xg, yg, bc, precision, "flow")
        if split:
            assert tune.set_split_level(s, split) and tune.split_level(s) == split
        s.set_state(*st)
        code, _, _ = s.dev.newton(0.3)
        assert code == 0, v2d._lib.last_error()
        out = np.concatenate(s.dev.get_state()[:2]) - np.concatenate(st[:2])
        nl = len(tune.item_rows(s))
        s.close()
        return out, nl

    ref, nl = update(0)
    scale = np.abs(ref).max()
    for split in sorted({1, min(3, nl - 1), nl - 1}):
        got, _ = update(split)
        assert np.max(np.abs(got - ref)) <= 1e-10 * scale, split
