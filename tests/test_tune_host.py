"""Host logic of the LU-solve autotuner (vorti2d_b200/tune.py) on a fake
solver: the device calls (item rows, kernel form, split level, timed
applications) are replaced by a synthetic cost model, so the coordinate
search, the gain threshold, the split search and the JSON record are checked
without a GPU."""
import json

import pytest

from vorti2d_b200 import tune


class FakeCfg:
    precision = "mixed"
    lu_factors = "fp32"


class FakeSolver:
    """Cost of one application: a separable function of the rows per item of
    each level, plus terms for the kernel form and the split level.  Split
    levels above `max_split` do not fit (the setter refuses them)."""

    def __init__(self, nlevel=6, best_rows=None, best_form=1, best_split=0, max_split=4):
        self.imax = self.jmax = 181
        self.cfg = FakeCfg()
        self.nlevel = nlevel
        self.rows = [16] * nlevel
        self.form = 0
        self.split = 0
        self.best_rows = best_rows or [0, -32, 64, 8, 8, 128][:nlevel]
        self.best_form = best_form
        self.best_split = best_split
        self.max_split = max_split
        self.timings = 0

    def cost(self):
        t = 1.0
        for L, (r, b) in enumerate(zip(self.rows, self.best_rows)):
            t += 0.02 * (0 if r == b else 1 + L % 3)   # each above the 1 % gain
        t += 0.0 if self.form == self.best_form else 0.05
        t += 0.0 if self.split == self.best_split else 0.03 * (1 + abs(self.split - self.best_split))
        return t


@pytest.fixture
def fake(monkeypatch):
    def install(solver):
        monkeypatch.setattr(tune, "item_rows", lambda s: list(s.rows))
        monkeypatch.setattr(tune, "set_item_rows",
                            lambda s, r: setattr(s, "rows", [int(v) for v in r]))
        monkeypatch.setattr(tune, "flow_form", lambda s: s.form)

        def set_form(s, f):
            s.form = int(f)
            return True
        monkeypatch.setattr(tune, "set_flow_form", set_form)
        monkeypatch.setattr(tune, "split_level", lambda s: s.split)

        def set_split(s, lv):
            if lv > s.max_split:
                return False
            s.split = int(lv)
            return True
        monkeypatch.setattr(tune, "set_split_level", set_split)

        def timed(s, reps=30, repeats=3):
            s.timings += 1
            return s.cost()
        monkeypatch.setattr(tune, "time_apply", timed)
        return solver
    return install


def test_search_finds_the_separable_optimum(fake):
    s = fake(FakeSolver())
    rec = tune.tune_lu_solve(s, reps=5)
    assert rec["rows"] == s.best_rows and s.rows == s.best_rows
    assert rec["form"] == 1 and s.form == 1
    assert rec["split"] == 0 and s.split == 0
    assert rec["ms"] == pytest.approx(1.0)
    assert rec["default_ms"] > rec["ms"]
    assert rec["key"] == "181x181/mixed/fp32"
    assert rec["trials"] > 0 and rec["reps"] == 5


def test_split_search_skips_levels_that_do_not_fit(fake):
    s = fake(FakeSolver(best_split=3, max_split=4))
    rec = tune.tune_lu_solve(s, reps=5)
    assert rec["split"] == 3 and s.split == 3
    # a split beyond what fits is never selected
    s2 = fake(FakeSolver(best_split=7, max_split=4))
    rec2 = tune.tune_lu_solve(s2, reps=5)
    assert rec2["split"] <= 4


def test_gain_threshold_keeps_the_default(fake):
    """Trials faster by less than `gain` do not replace the current choice."""
    s = fake(FakeSolver())
    start = list(s.rows)
    rec = tune.tune_lu_solve(s, reps=5, gain=0.5)
    assert rec["rows"] == start and rec["form"] == 0 and rec["split"] == 0
    assert rec["ms"] == rec["default_ms"]


def test_record_merges_into_the_json_file_and_reloads(fake, tmp_path):
    path = str(tmp_path / "tuning.json")
    with open(path, "w") as fh:
        json.dump({"other/key": {"rows": [1, 2]}}, fh)
    s = fake(FakeSolver(best_split=2))
    rec = tune.tune_lu_solve(s, reps=5, path=path)
    with open(path) as fh:
        table = json.load(fh)
    assert set(table) == {"other/key", rec["key"]}
    assert table[rec["key"]]["rows"] == rec["rows"]
    # a fresh solver of the same grid and precision picks the record up
    s2 = fake(FakeSolver(best_split=2))
    assert tune.load_tuning(s2, path)
    assert s2.rows == rec["rows"] and s2.form == rec["form"] and s2.split == rec["split"]


def test_load_tuning_rejects_missing_or_mismatched_records(fake, tmp_path):
    s = fake(FakeSolver())
    assert not tune.load_tuning(s, str(tmp_path / "absent.json"))
    path = str(tmp_path / "t.json")
    with open(path, "w") as fh:
        json.dump({"181x181/mixed/fp32": {"rows": [0, 8]}}, fh)   # wrong level count
    before = list(s.rows)
    assert not tune.load_tuning(s, path)
    assert s.rows == before
