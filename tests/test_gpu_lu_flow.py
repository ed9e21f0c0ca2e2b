"""The dataflow solve of the LU preconditioner's upper levels (opt-in:
V2D_LU_FLOW=1 when the factors are created) against the per-phase launches.
It runs the same item functions in another schedule and each output entry is
written by one item, so the Newton updates agree bit for bit.  These tests
run only with V2D_TEST_LU_FLOW=1, while the dataflow solve stays opt-in."""
import ctypes
import os

import numpy as np
import pytest

from cases import smooth_state

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("V2D_TEST_LU_FLOW") != "1",
                                 reason="the dataflow LU solve is opt-in (V2D_TEST_LU_FLOW=1)")]

SHAPES = [(9, 7, 1), (33, 21, 1), (64, 48, 0), (129, 65, 2), (181, 181, 1)]


def _solver(v2d, xg, yg, bc, precision, flow, monkeypatch):
    if flow:
        monkeypatch.setenv("V2D_LU_FLOW", "1")
    else:
        monkeypatch.delenv("V2D_LU_FLOW", raising=False)
    cfg = v2d.Config(verbose=False, write_csv=False, write_xdmf=False, compute_forces=False,
                     re=80.0, steady=False, dt_phys=0.2, farfield_bc=bc, alpha_deg=4.0,
                     precision=precision, precond="lu", ksp_rtol=1e-12)
    return v2d.Solver(cfg, mesh=(xg, yg))


@pytest.mark.parametrize("imax,jmax,ff_bc", SHAPES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_flow_newton_update_equals_per_phase(v2d, oracle_mod, monkeypatch, imax, jmax, ff_bc,
                                             precision):
    bc = {0: "dirichlet", 1: "outflow", 2: "outflow_psi"}[ff_bc]
    xg, yg = oracle_mod.generate_cylinder(imax, jmax)
    M = oracle_mod.core().compute_metrics(1 / (imax - 1), 1 / (jmax - 1), xg, yg)
    st = smooth_state(M[8], M[9])
    out = []
    for flow in (False, True):
        s = _solver(v2d, xg, yg, bc, precision, flow, monkeypatch)
        s.set_state(*st)
        code, res, lin = s.dev.newton(0.3)
        assert code == 0, v2d._lib.last_error()
        out.append((np.concatenate(s.dev.get_state()[:2]), lin.iterations, res))
        s.close()
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][2] == out[1][2]


def test_flow_launch_list_181(v2d, oracle_mod, monkeypatch):
    """181x181: the solve becomes 9 launches (4 one-CTA-per-front levels up,
    one dataflow launch, 4 down) and its device time is printed beside the
    per-phase solve's."""
    from vorti2d_b200 import _lib
    xg, yg = oracle_mod.generate_cylinder(181, 181)
    M = oracle_mod.core().compute_metrics(1 / 180, 1 / 180, xg, yg)
    st = smooth_state(M[8], M[9])
    totals = []
    for flow in (False, True):
        s = _solver(v2d, xg, yg, "outflow", "mixed", flow, monkeypatch)
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
        if flow:
            assert n.value == 9 and kinds.count(6) == 1, kinds
        else:
            assert n.value == 34 and 6 not in kinds, kinds
        totals.append(sum(ms[k] for k in range(n.value)))
        s.close()
    print(f"LU solve 181x181 mixed, warm: per-phase {totals[0]:.3f} ms, "
          f"dataflow {totals[1]:.3f} ms")
