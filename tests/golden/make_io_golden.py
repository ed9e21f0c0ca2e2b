"""Write the file-format fixtures under tests/golden/ref_io/ with the
reference's own writers (vorti2d/restart.py, vorti2d/fields_io.py), loaded
unmodified by file path (they import only numpy):

    python tests/golden/make_io_golden.py /path/to/vorti2d-reference

The state is a small seeded one (5x4 grid) so the fixtures stay a few KB.
tests/test_io_formats.py reads them back with vorti2d_b200's readers and
compares vorti2d_b200's writers with them byte for byte.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "ref_io")
IMAX, JMAX = 5, 4
FORCE_COLUMNS = ("t", "cd", "cl", "cm", "cdp", "cdf", "clp", "clf", "cmp", "cmf")


def load(ref_root, name):
    path = os.path.join(ref_root, "vorti2d", name + ".py")
    spec = importlib.util.spec_from_file_location("refio_" + name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def sample_state(seed=7):
    """Seeded state, grid and per-step records used by the fixtures and the
    test (the test rebuilds them with the same seed)."""
    rng = np.random.default_rng(seed)
    n = IMAX * JMAX
    fields = [rng.standard_normal(n) * 10.0 ** rng.integers(-3, 3) for _ in range(4)]
    fields[0][3] = -0.0                      # a signed zero must survive the text format
    xg = rng.standard_normal((IMAX, JMAX))
    yg = rng.standard_normal((IMAX, JMAX))
    res_log = list(np.log10(np.abs(rng.standard_normal(6)) * 1e-4))
    rows = [{c: float(v) for c, v in zip(FORCE_COLUMNS, rng.standard_normal(10))}
            for _ in range(3)]
    return fields, xg, yg, res_log, rows


def main(ref_root):
    restart = load(ref_root, "restart")
    fio = load(ref_root, "fields_io")
    fields, xg, yg, res_log, rows = sample_state()
    os.makedirs(OUT, exist_ok=True)
    restart.save_restart(os.path.join(OUT, "restart.npz"),
                         restart.RestartState(*fields, 12.4, 62, IMAX, JMAX, 100.0))
    fio.ensure_dirs(OUT)
    fio.write_grid(OUT, xg, yg)
    fio.write_fields(OUT, 62, fields[0], fields[1])
    fio.write_residual_history(OUT, 62, res_log)
    fio.init_force_history(OUT, FORCE_COLUMNS)
    for r in rows:
        fio.append_force_history(OUT, FORCE_COLUMNS, r)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VORTI2D_REFERENCE", "../reference"))
