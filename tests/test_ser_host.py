"""Control logic of the pseudo-transient continuation
(vorti2d_b200.adjoint.steady_solve_ser) on a scripted fake device: dtau
growth, the switched-evolution-relaxation bound, the undo of a blow-up, the
halving after a rise, the floor on dtau and the restored 1/dtau of the
handle (CPU only)."""
import math

import numpy as np
import pytest

from vorti2d_b200 import _lib, adjoint


class FakeParams:
    invdtau = 0.0


class FakeDev:
    """State: one marker x.  Each Newton call moves to the next scripted
    marker and reports the scripted update norm; the residual norm of a
    marker comes from a table."""

    def __init__(self, steps):
        self.x = 0
        self.steps = list(steps)
        self.params = FakeParams()
        self.invdtau_seen = []
        self.x_seen = []

    def get_state(self):
        return [np.array([self.x])]

    def set_state(self, x):
        self.x = int(x[0])

    def set_invdtau(self, v):
        self.params.invdtau = v
        self.invdtau_seen.append(v)

    def newton(self, urot):
        self.x_seen.append(self.x)
        step = self.steps.pop(0)
        if isinstance(step, Exception):
            raise step
        self.x, res = step
        return _lib.V2D_OK, res, None


class FakeCfg:
    pseudo_tol = 1e-10
    re = 40.0
    alpha_deg = 0.0

    def u_rot(self, t):
        return 0.0


class FakeSolver:
    def __init__(self, dev):
        self.dev, self.cfg, self._host_state = dev, FakeCfg(), None


@pytest.fixture
def residuals(monkeypatch):
    table = {}
    monkeypatch.setattr(adjoint, "_residual",
                        lambda solver, re, adeg, urot: np.array([table[solver.dev.x]]))
    return table


def test_growth_rejection_and_halving(residuals):
    residuals.update({0: 1.0, 1: 0.5, 2: 0.1, 3: 1e6, 4: 0.2, 5: 1e-3})
    dev = FakeDev([(1, 1e-2), (2, 1e-3), (3, 1e2), (4, 1e-4), (5, 1e-12)])
    dev.params.invdtau = 0.125
    res, it = adjoint.steady_solve_ser(FakeSolver(dev), dtau0=1.0, growth=2.0, reject=1e3)
    assert res == 1e-12 and it == 5
    # dtau: 1; 2 (growth, SER bound 2); 10 (SER bound 1 * 1.0 / 0.1 above
    # growth); the blow-up to 1e6 is undone and quarters dtau to 2.5; the rise
    # to 0.2 halves it to 1.25; then the last step
    want = [1.0, 1 / 2.0, 1 / 10.0, 1 / 2.5, 1 / 1.25]
    assert dev.invdtau_seen[:5] == pytest.approx(want)
    # the rejected step's state was restored before the next Newton call
    assert dev.x_seen == [0, 1, 2, 2, 4]
    # the handle's own 1/dtau is back
    assert dev.params.invdtau == 0.125 and dev.invdtau_seen[-1] == 0.125


def test_repeated_blowups_stop_at_the_dtau_floor(residuals):
    residuals.update({0: 1.0, 9: 1e9})
    dev = FakeDev([(9, 1.0)] * 10)
    res, it = adjoint.steady_solve_ser(FakeSolver(dev), dtau0=1.0)
    # dtau 1 -> 1/4 -> 1/16 -> 1/64 (the floor dtau0 / 64), then the next
    # rejection at the floor stops the loop
    assert math.isinf(res) and it == 4
    assert dev.invdtau_seen[:4] == pytest.approx([1.0, 4.0, 16.0, 64.0])
    assert dev.x == 0   # every step undone


def test_non_finite_update_counts_as_a_failed_step(residuals):
    residuals.update({0: 1.0, 1: 0.5, 2: 0.01})
    dev = FakeDev([(1, float("nan")), (2, 1e-12)])
    res, it = adjoint.steady_solve_ser(FakeSolver(dev), dtau0=4.0)
    assert res == 1e-12 and it == 2
    assert dev.x_seen == [0, 0]   # the NaN step was undone
    assert dev.invdtau_seen[:2] == pytest.approx([1 / 4.0, 1 / 1.0])


def test_invdtau_restored_when_newton_raises(residuals):
    residuals.update({0: 1.0})
    dev = FakeDev([RuntimeError("device error")])
    dev.params.invdtau = 0.5
    with pytest.raises(RuntimeError):
        adjoint.steady_solve_ser(FakeSolver(dev), dtau0=1.0)
    assert dev.params.invdtau == 0.5


def test_max_iter_bounds_the_loop(residuals):
    residuals.update({0: 1.0, 1: 0.9, 2: 0.8, 3: 0.7})
    dev = FakeDev([(1, 1.0), (2, 1.0), (3, 1.0)])
    res, it = adjoint.steady_solve_ser(FakeSolver(dev), dtau0=1.0, max_iter=3)
    assert it == 3 and res == 1.0


def test_rejected_step_with_a_small_update_is_not_reported_converged(residuals):
    """A blow-up undone at the dtau floor leaves the state before it: its own
    update norm, however small, is not the result."""
    residuals.update({0: 1.0, 9: 1e9})
    dev = FakeDev([(9, 1e-14)] * 10)
    res, it = adjoint.steady_solve_ser(FakeSolver(dev), dtau0=1.0, tol=1e-10)
    assert math.isinf(res) and it == 4 and dev.x == 0
