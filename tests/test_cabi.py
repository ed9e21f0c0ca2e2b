"""The C-ABI library without a GPU: it builds, loads, exports every entry
point that include/vorti2d_b200.h declares, and its host-only paths (argument
checks, defaults, neighbour indices) behave as documented.  No call here
launches a kernel."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "include")


def declared_symbols():
    names = set()
    for fn in os.listdir(HEADER_DIR):
        if fn.endswith(".h"):
            text = open(os.path.join(HEADER_DIR, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names.update(re.findall(r"\b(v2d_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib(v2d):
    from vorti2d_b200 import _lib
    return ctypes.CDLL(_lib.LIB_PATH)


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(v2d):
    from vorti2d_b200 import _lib
    bound = set(_lib._SIGS)
    missing = [n for n in declared_symbols() if n not in bound]
    assert not missing, missing


def test_library_is_built_for_sm100a(v2d):
    """The in-tree library carries sm_100a code (fatbin section present)."""
    from vorti2d_b200 import _lib
    data = open(_lib.LIB_PATH, "rb").read()
    assert b".nv_fatbin" in data or b"__nv_relfatbin" in data
    assert b"sm_100a" in data


def test_host_only_entry_points(v2d):
    from vorti2d_b200 import _lib
    L = _lib.lib()
    assert L.v2d_version() >= 10000
    p = _lib.KrylovParams()
    L.v2d_krylov_defaults(ctypes.byref(p))
    assert p.restart == 30 and p.rtol == 1e-10 and p.precond == _lib.PC_BJACOBI
    out = (ctypes.c_int * 9)()
    assert L.v2d_node_neighbors(1, 2, 9, out) == 0
    # i=1 wraps west to i=imax-1 (vorti2d_core.f90:39-52)
    k = 9 * 1 + 1
    assert list(out) == [k, k + 1, k + 7, k + 9, k - 9, k + 10, k + 16, k - 8, k - 2]
    assert L.v2d_node_neighbors(0, 2, 9, out) == _lib.V2D_EARG
    assert b"node_neighbors" in L.v2d_last_error()


def test_krylov_defaults_and_config_mapping(v2d):
    """The C defaults factor every Newton Jacobian (as MUMPS does) and keep
    no factors across steps; Config's GPU knobs reach the C structure."""
    from vorti2d_b200 import _lib
    from vorti2d_b200.solver import solver_params
    d = _lib.krylov_defaults()
    assert d.lu_reuse_its == 0 and d.lu_reuse_steps == 0 and d.lu_leaf == 64
    p = solver_params(v2d.Config(re=150.0, precision="mixed", precond="lu", lu_reuse_its=12,
                                 lu_reuse_steps=True, krylov_max_it=300))
    assert p.re == 150.0 and p.krylov.lu_reuse_its == 12 and p.krylov.lu_reuse_steps == 1
    assert p.krylov.precond == _lib.PC_LU and p.krylov.precision == _lib.PREC_MIXED
    assert p.krylov.max_it == 300
    q = solver_params(v2d.Config())
    assert q.krylov.lu_reuse_its == 0 and q.krylov.lu_reuse_steps == 0


def test_argument_errors_before_any_device_work(v2d):
    from vorti2d_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    prm = _lib.SolverParams()
    assert L.v2d_solver_create(181, 181, None, None, ctypes.byref(prm), ctypes.byref(h)) \
        == _lib.V2D_EARG
    assert L.v2d_solver_destroy(None) == 0
    # handle-based entry points reject a null handle before any device work
    n = ctypes.c_int()
    ms = (ctypes.c_double * 4)()
    codes = (ctypes.c_int * 4)()
    b = (ctypes.c_double * 8)()
    x = (ctypes.c_double * 4)()
    assert L.v2d_solver_time_lu_launches(None, 1, 0, ms, codes, 4, ctypes.byref(n)) \
        == _lib.V2D_EARG
    assert L.v2d_solver_time_lu_factor(None, 1, ms, codes, 4, ctypes.byref(n)) == _lib.V2D_EARG
    assert L.v2d_solver_residual_mesh(None, x, x, 40.0, 0.0, 0.0, 0.0, 1.0, 0.0, b, 0,
                                      None) == _lib.V2D_EARG
    assert "null" in _lib.last_error()


def handle_entry_points():
    """(name, argument count) of every declared function whose first
    parameter is a solver, linear-system or batch handle."""
    out = []
    for fn in os.listdir(HEADER_DIR):
        if not fn.endswith(".h"):
            continue
        text = re.sub(r"/\*.*?\*/", "", open(os.path.join(HEADER_DIR, fn)).read(), flags=re.S)
        for m in re.finditer(r"^int (v2d_\w+)\(([^;]*?)\);", text, re.M | re.S):
            params = " ".join(m.group(2).split())
            if re.match(r"(const )?v2d_(solver|linsys|batch) \*", params):
                out.append((m.group(1), params.count(",") + 1))
    return sorted(out)


@pytest.mark.parametrize("name,nargs", handle_entry_points())
def test_null_handle_is_an_argument_error(v2d, name, nargs):
    """Every entry point taking a handle rejects a null one with V2D_EARG
    before touching the device (the destroy calls accept null, as free
    does)."""
    from vorti2d_b200 import _lib
    f = getattr(_lib.lib(), name)
    types = f.argtypes or []
    args = []
    for k in range(nargs):
        t = types[k] if k < len(types) else ctypes.c_void_p
        if t in (ctypes.c_int, ctypes.c_uint, ctypes.c_long, ctypes.c_longlong, ctypes.c_size_t):
            args.append(0)
        elif t in (ctypes.c_double, ctypes.c_float):
            args.append(0.0)
        else:
            args.append(None)
    code = f(*args)
    if name.endswith("_destroy"):
        assert code == _lib.V2D_OK
    else:
        assert code == _lib.V2D_EARG, (name, code, _lib.last_error())


def value_entry_points():
    """(name, argument count) of every declared function that takes no
    handle and has arguments."""
    out = []
    for fn in os.listdir(HEADER_DIR):
        if not fn.endswith(".h"):
            continue
        text = re.sub(r"/\*.*?\*/", "", open(os.path.join(HEADER_DIR, fn)).read(), flags=re.S)
        for m in re.finditer(r"^int (v2d_\w+)\(([^;]*?)\);", text, re.M | re.S):
            params = " ".join(m.group(2).split())
            if params in ("", "void") or re.match(r"(const )?v2d_(solver|linsys|batch) \*", params):
                continue
            out.append((m.group(1), params.count(",") + 1))
    return sorted(out)


@pytest.mark.parametrize("sizes", [(0, 0), (9, 7)])
@pytest.mark.parametrize("name,nargs", value_entry_points())
def test_null_arrays_are_an_argument_error(v2d, name, nargs, sizes):
    """Entry points without a handle reject zero sizes, and null arrays at
    valid sizes, with V2D_EARG and a message, before any device work."""
    from vorti2d_b200 import _lib
    f = getattr(_lib.lib(), name)
    types = f.argtypes or []
    args = []
    for k in range(nargs):
        t = types[k] if k < len(types) else ctypes.c_void_p
        if t in (ctypes.c_int, ctypes.c_uint, ctypes.c_long, ctypes.c_longlong, ctypes.c_size_t):
            args.append(sizes[k] if k < 2 else 0)
        elif t in (ctypes.c_double, ctypes.c_float):
            args.append(0.0)
        else:
            args.append(None)
    assert f(*args) == _lib.V2D_EARG, name
    assert _lib.last_error()


def test_handle_entry_points_are_found():
    names = [n for n, _ in handle_entry_points()]
    assert len(names) >= 40
    assert {"v2d_solver_newton", "v2d_linsys_solve", "v2d_batch_newton"} <= set(names)


def test_no_cpu_fallback(v2d, monkeypatch, tmp_path):
    """A missing library raises instead of falling back to another path."""
    from vorti2d_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_LIB", None, raising=False)
    with pytest.raises((RuntimeError, OSError)):
        _lib.lib()
