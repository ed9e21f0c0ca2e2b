"""Host logic of the batched steady sweep: the Reynolds continuation ladder
and the per-instance Newton loop, driven by a fake solver on the CPU."""
import math
from types import SimpleNamespace

import pytest

from vorti2d_b200.batch import CaseResult, re_ladder, solve_case


def test_ladder_without_continuation_is_the_target():
    assert re_ladder(300.0, 80.0, None) == [300.0]
    assert re_ladder(300.0, 80.0, 0) == [300.0]
    assert re_ladder(60.0, 80.0, 1.5) == [60.0]
    assert re_ladder(80.0, 80.0, 1.5) == [80.0]


def test_ladder_geometric_then_target():
    lad = re_ladder(1000.0, 80.0, 1.5)
    assert lad[0] == 80.0 and lad[-1] == 1000.0
    assert all(b > a for a, b in zip(lad, lad[1:]))
    assert all(b / a == pytest.approx(1.5) for a, b in zip(lad[:-2], lad[1:-1]))
    assert lad[-2] < 1000.0 <= lad[-2] * 1.5


@pytest.mark.parametrize("bad", [(math.nan, 80.0, 1.5), (-5.0, 80.0, 1.5), (300.0, 80.0, 0.9),
                                 (300.0, 80.0, math.inf), (300.0, -1.0, 1.5)])
def test_ladder_rejects_bad_arguments(bad):
    with pytest.raises(ValueError):
        re_ladder(*bad)


class FakeSolver:
    """Newton update norms scripted per Reynolds number: each call returns the
    next entry of ``script[re]``."""

    def __init__(self, re, script):
        self.re = re
        self.script = {k: list(v) for k, v in script.items()}
        self.set_calls = []
        self.cfg = SimpleNamespace(u_rot=lambda t: 0.0, t_start=0.0, inv_dtau=lambda: 0.0,
                                   inv_2dt=lambda: 0.0)
        self.dev = SimpleNamespace(set_re=self._set_re)
        self._last_lin = SimpleNamespace(iterations=3)

    def _set_re(self, re):
        self.set_calls.append(re)
        self.re = re

    def _assemble_and_solve_once(self, invdtau, inv2dt, urot):
        return self.script[self.re].pop(0)


def _case():
    return CaseResult("c", 300.0, 0.0, 100, False, 0, math.inf)


def test_plain_newton_converges_without_touching_re():
    s = FakeSolver(300.0, {300.0: [1e-2, 1e-5, 1e-11]})
    r = _case()
    res = solve_case(s, r, [300.0], 20, 1e-10, 1e-7, 1e3)
    assert res == 1e-11 and r.converged and not r.diverged
    assert r.newton_iters == 3 and r.krylov_iters == 9 and r.rungs == 1
    assert r.re_reached == 300.0 and s.set_calls == []


def test_continuation_walks_the_ladder_with_rung_tolerance():
    s = FakeSolver(80.0, {80.0: [1e-2, 1e-8], 120.0: [1e-3, 5e-8], 300.0: [1e-3, 1e-8, 1e-11]})
    r = _case()
    solve_case(s, r, [80.0, 120.0, 300.0], 20, 1e-10, 1e-7, 1e3)
    assert r.converged and s.set_calls == [80.0, 120.0, 300.0]
    assert r.newton_iters == 7 and r.rungs == 3 and r.re_reached == 300.0


def test_failed_rung_stops_and_reports_the_last_reached():
    s = FakeSolver(80.0, {80.0: [1e-8], 120.0: [1e-3] * 4})
    r = _case()
    res = solve_case(s, r, [80.0, 120.0, 300.0], 4, 1e-10, 1e-7, 1e3)
    assert not r.converged and not r.diverged and res == 1e-3
    assert r.re_reached == 80.0 and r.rungs == 2 and r.newton_iters == 5


def test_divergence_and_nonfinite_updates_stop_the_instance():
    s = FakeSolver(300.0, {300.0: [1e-3, 2.0]})
    r = _case()
    solve_case(s, r, [300.0], 20, 1e-10, 1e-7, 1e3)
    assert r.diverged and not r.converged and r.newton_iters == 2
    s = FakeSolver(300.0, {300.0: [1e-3, math.nan]})
    r = _case()
    solve_case(s, r, [300.0], 20, 1e-10, 1e-7, 1e3)
    assert r.diverged and not r.converged and math.isnan(r.re_reached)


def test_small_update_that_grows_a_thousandfold_is_diverged():
    s = FakeSolver(300.0, {300.0: [1e-9, 1e-5]})
    r = _case()
    solve_case(s, r, [300.0], 20, 1e-10, 1e-7, 1e3)
    assert r.diverged and not r.converged
