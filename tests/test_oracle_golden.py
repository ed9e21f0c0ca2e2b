"""The oracle and the host-side mirrors against golden vectors made by the
reference's own pure-NumPy modules (tests/golden/make_golden.py): the
cylinder generator (vorti2d/mesh.py:14-50), the force integrals
(vorti2d/forces.py:82-194) and the Config scalars (vorti2d/config.py:139-166).
"""
import hashlib
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "reference_golden.npz")
FORCE_OPTS = [(None, (0.0, 0.0)), (1.0, (0.25, -0.1)), (2.5, (-0.3, 0.7))]
CONFIGS = [
    dict(),
    dict(re=40.0, steady=True, rot_speed=0.5),
    dict(re=100.0, dt_phys=0.2, rot_speed=0.5, rot_until=2.0, farfield_bc="outflow"),
    dict(re=500.0, steady=True, alpha_deg=4.0, farfield_bc="outflow_psi", dtau=2.0),
    dict(re=80.0, dt_phys=0.05, alpha_deg=-8.0, farfield_bc="Dirichlet", dtau=0.5),
]
U_ROT_TIMES = [0.0, 0.2, 1.9, 2.0, 2.0000001, 5.0]
FORCE_KEYS = ("cd", "cl", "cm", "cdp", "cdf", "clp", "clf", "cmp", "cmf", "ref_length")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def _mesh_keys(golden):
    out = []
    for k in golden.files:
        if k.startswith("mesh_") and k.endswith("_x"):
            dims, ri, ro = k[5:-2].split("_")
            im, jm = (int(v) for v in dims.split("x"))
            out.append((k[:-2], im, jm, float(ri), float(ro)))
    return out


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_cylinder_generator_bit_exact(golden, oracle_mod, which):
    if which == "oracle":
        gen = oracle_mod.generate_cylinder
    else:
        from vorti2d_b200.mesh import generate_cylinder as gen
    keys = _mesh_keys(golden)
    assert len(keys) >= 4
    for key, im, jm, ri, ro in keys:
        xg, yg = gen(im, jm, ri, ro)
        assert xg.shape == (im, jm)
        assert np.array_equal(xg, golden[key + "_x"]), key
        assert np.array_equal(yg, golden[key + "_y"]), key
    for tag, hx, hy in golden["mesh_hashes"]:
        dims, ri, ro = str(tag).split("_")
        im, jm = (int(v) for v in dims.split("x"))
        xg, yg = gen(im, jm, float(ri), float(ro))
        assert _sha(xg) == hx and _sha(yg) == hy, tag


@pytest.mark.parametrize("mesh", ["25x17", "65x49"])
@pytest.mark.parametrize("field", ["sym", "asym"])
def test_force_coeffs_match_reference(golden, oracle_mod, mesh, field):
    im, jm = (int(v) for v in mesh.split("x"))
    key = f"forces_{mesh}"
    g = {n: golden[f"{key}_in_{n}"] for n in ("beta", "gama", "detadx", "detady", "xphys",
                                              "yphys")}
    ome = golden[f"{key}_in_ome_{field}"]
    want = golden[f"{key}_out_{field}"]
    for row, (ref_length, mref) in zip(want, FORCE_OPTS):
        fc = oracle_mod.compute_force_coeffs(im, jm, 40.0, 1.0 / (im - 1), 1.0 / (jm - 1),
                                             g["beta"], g["gama"], g["detadx"], g["detady"],
                                             g["xphys"], g["yphys"], ome,
                                             ref_length=ref_length, moment_ref=mref)
        scale = max(abs(row[3]), abs(row[4]), abs(row[7]), abs(row[8]))
        for k, w in zip(FORCE_KEYS, row):
            assert abs(getattr(fc, k) - w) <= 1e-12 * max(scale, abs(w)), (k, getattr(fc, k), w)


def test_force_columns(golden, oracle_mod):
    from vorti2d_b200.forces import FORCE_COLUMNS
    ref = tuple(str(c) for c in golden["force_columns"])
    assert oracle_mod.FORCE_COLUMNS == ref
    assert FORCE_COLUMNS == ref


def test_config_scalars_match_reference(golden, oracle_mod):
    from vorti2d_b200 import Config
    for kw, row in zip(CONFIGS, golden["config_scalars"]):
        c = Config(**kw)
        got = [c.inv_dtau(), c.inv_2dt(), c.cos_alpha(), c.sin_alpha(), float(c.ff_bc_code())]
        got += [c.u_rot(t) for t in U_ROT_TIMES]
        assert np.array_equal(np.array(got), row), kw
        o = oracle_mod.config_scalars(kw.get("re", 60.0), kw.get("steady", False),
                                      kw.get("dt_phys", 0.2), kw.get("dtau", math.inf),
                                      kw.get("alpha_deg", 0.0), kw.get("farfield_bc",
                                                                       "dirichlet"))
        assert np.array_equal(np.array(o, dtype=float), row[:5]), kw
        ur = [oracle_mod.u_rot(t, kw.get("steady", False), kw.get("rot_speed", 0.0),
                               kw.get("rot_until", 0.0)) for t in U_ROT_TIMES]
        assert np.array_equal(np.array(ur), row[5:]), kw


def test_config_is_a_drop_in(golden):
    """Every field of the reference Config exists with the same default; the
    GPU knobs come after them, all defaulted."""
    import dataclasses
    from vorti2d_b200 import Config
    fields = dataclasses.fields(Config)
    ref = [(str(n), str(d)) for n, d in golden["config_fields"]]
    assert [(f.name, repr(f.default)) for f in fields[:len(ref)]] == ref
    for f in fields[len(ref):]:
        assert f.default is not dataclasses.MISSING, f.name
    with pytest.raises(ValueError):
        Config(farfield_bc="bogus").ff_bc_code()


@pytest.mark.parametrize("mesh", ["25x17", "65x49"])
def test_velocity_matches_reference(golden, oracle_mod, mesh):
    """vorti2d/velocity.py:76-93 restated: bit-exact with the reference's
    NumPy evaluation on the same metrics and streamfunction."""
    im, jm = (int(v) for v in mesh.split("x"))
    key = f"velocity_{mesh}"
    g = {n: golden[f"{key}_in_{n}"] for n in ("jac", "beta", "gama", "detadx", "detady", "psi")}
    u, v, mag = oracle_mod.compute_velocity(im, jm, 1.0 / (im - 1), 1.0 / (jm - 1), g["jac"],
                                            g["beta"], g["gama"], g["detadx"], g["detady"],
                                            g["psi"], want_mag=True)
    want = golden[f"{key}_out"]
    assert np.array_equal(u, want[0]) and np.array_equal(v, want[1])
    assert np.array_equal(mag, want[2])
