"""File formats of vorti2d_b200's run output and checkpoints against files the
reference's own writers produced (tests/golden/ref_io/, from
tests/golden/make_io_golden.py): a reference checkpoint loads into the same
state, and every text file vorti2d_b200 writes for the same data is
byte-identical to the reference's."""
import filecmp
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
REF = os.path.join(HERE, "golden", "ref_io")

from make_io_golden import FORCE_COLUMNS, IMAX, JMAX, sample_state  # noqa: E402


def test_reference_checkpoint_loads():
    from vorti2d_b200 import restart
    fields, *_ = sample_state()
    st = restart.load_restart(os.path.join(REF, "restart.npz"), IMAX, JMAX)
    for name, want in zip(restart.FIELDS, fields):
        got = getattr(st, name)
        assert got.dtype == np.float64 and np.array_equal(got, want)
    assert np.signbit(st.psi[3])
    assert (st.t, st.step, st.imax, st.jmax, st.re) == (12.4, 62, IMAX, JMAX, 100.0)
    assert isinstance(st.step, int) and isinstance(st.t, float)
    with pytest.raises(ValueError, match="restart mesh"):
        restart.load_restart(os.path.join(REF, "restart.npz"), IMAX + 1, JMAX)


def test_checkpoint_round_trip_has_reference_members(tmp_path):
    from vorti2d_b200 import restart
    fields, *_ = sample_state()
    p = restart.save_restart(str(tmp_path / "r"), restart.RestartState(
        *fields, 12.4, 62, IMAX, JMAX, 100.0))
    assert p.endswith("r.npz") and os.path.exists(p)
    with np.load(p) as mine, np.load(os.path.join(REF, "restart.npz")) as ref:
        assert sorted(mine.files) == sorted(ref.files)
        for k in ref.files:
            assert mine[k].dtype == ref[k].dtype and mine[k].shape == ref[k].shape, k
            assert np.array_equal(mine[k], ref[k]), k
    assert not [f for f in os.listdir(tmp_path) if f.startswith(".restart-")]


def test_text_output_is_byte_identical(tmp_path):
    from vorti2d_b200 import fields_io
    fields, xg, yg, res_log, rows = sample_state()
    out = str(tmp_path)
    fields_io.ensure_dirs(out)
    fields_io.write_grid(out, xg, yg)
    fields_io.write_fields(out, 62, fields[0], fields[1])
    fields_io.write_residual_history(out, 62, res_log)
    fields_io.init_force_history(out, FORCE_COLUMNS)
    for r in rows:
        fields_io.append_force_history(out, FORCE_COLUMNS, r)
    rel = ["xg.csv", "yg.csv", "forces.csv", "psi_data/psi_t0062.csv",
           "omega_data/omega_t0062.csv", "residual_data/residual_history_t0062.csv"]
    for f in rel:
        assert filecmp.cmp(os.path.join(out, f), os.path.join(REF, f), shallow=False), f
