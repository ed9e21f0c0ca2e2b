"""Generate the golden vectors in this folder from the reference's own
pure-NumPy modules (run in a checkout that has the reference next to it):

    python tests/golden/make_golden.py /path/to/vorti2d-reference

The reference's Fortran core and PETSc layer cannot be built without a Fortran
compiler and petsc4py, but ``vorti2d/mesh.py``, ``vorti2d/forces.py``,
``vorti2d/config.py`` and ``vorti2d/velocity.py`` import only numpy, so they
are loaded unmodified by file path and run here.  Their outputs pin the
oracle's restatements (mesh generator, force integrals, configuration
scalars, velocity reconstruction) and the product's kernels and host-side
mirrors of them.

Forces and velocities need metric arrays as input; those come from the
oracle's C restatement of ``compute_metrics`` and are stored next to the
outputs, so the golden values depend only on the reference's modules.
"""
from __future__ import annotations

import hashlib
import importlib.util
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MESHES_FULL = [(5, 4, 0.5, 50.0), (9, 7, 0.5, 50.0), (25, 17, 0.5, 50.0), (41, 41, 0.5, 50.0)]
MESHES_HASHED = [(121, 121, 0.5, 50.0), (129, 129, 0.5, 50.0), (181, 181, 0.5, 50.0),
                 (101, 151, 0.5, 100.0), (513, 513, 0.5, 50.0)]
FORCE_MESHES = [(25, 17), (65, 49)]
FORCE_OPTS = [(None, (0.0, 0.0)), (1.0, (0.25, -0.1)), (2.5, (-0.3, 0.7))]
CONFIGS = [
    dict(),
    dict(re=40.0, steady=True, rot_speed=0.5),
    dict(re=100.0, dt_phys=0.2, rot_speed=0.5, rot_until=2.0, farfield_bc="outflow"),
    dict(re=500.0, steady=True, alpha_deg=4.0, farfield_bc="outflow_psi", dtau=2.0),
    dict(re=80.0, dt_phys=0.05, alpha_deg=-8.0, farfield_bc="Dirichlet", dtau=0.5),
]
U_ROT_TIMES = [0.0, 0.2, 1.9, 2.0, 2.0000001, 5.0]


def load(ref_root, name):
    path = os.path.join(ref_root, "vorti2d", name + ".py")
    spec = importlib.util.spec_from_file_location("refmod_" + name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod          # dataclasses look their module up here
    spec.loader.exec_module(mod)
    return mod


def smooth_state(x, y):
    """Analytic state of the reference's tests/test_assemble_local.py:23-30."""
    r = np.sqrt(x ** 2 + y ** 2)
    psi = np.sin(0.3 * x) * np.cos(0.2 * y) / (1.0 + 0.01 * r)
    ome = np.cos(0.25 * x) * np.sin(0.15 * y) * np.exp(-0.02 * r)
    return psi, ome


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def main(ref_root):
    mesh = load(ref_root, "mesh")
    forces = load(ref_root, "forces")
    config = load(ref_root, "config")
    from oracle import oracle as O
    out = {}
    for (im, jm, ri, ro) in MESHES_FULL:
        xg, yg = mesh.generate_cylinder(im, jm, ri, ro)
        out[f"mesh_{im}x{jm}_{ri}_{ro}_x"] = xg
        out[f"mesh_{im}x{jm}_{ri}_{ro}_y"] = yg
    hashes = []
    for (im, jm, ri, ro) in MESHES_HASHED:
        xg, yg = mesh.generate_cylinder(im, jm, ri, ro)
        hashes.append([f"{im}x{jm}_{ri}_{ro}", sha(xg), sha(yg)])
    out["mesh_hashes"] = np.array(hashes)
    for (im, jm) in FORCE_MESHES:
        xg, yg = mesh.generate_cylinder(im, jm, 0.5, 50.0)
        dk, de = 1.0 / (im - 1), 1.0 / (jm - 1)
        M = O.core().compute_metrics(dk, de, xg, yg)
        _, ome = smooth_state(M[8], M[9])
        # a second, asymmetric field so that lift and moment are not zero
        ome_asym = ome + 0.5 * np.cos(0.3 * M[8] + 0.2 * M[9]) * np.exp(-0.05 * M[9] ** 2)
        key = f"forces_{im}x{jm}"
        for name, a in zip(("beta", "gama", "detadx", "detady", "xphys", "yphys"),
                           (M[2], M[3], M[6], M[7], M[8], M[9])):
            out[f"{key}_in_{name}"] = a
        for tag, field in (("sym", ome), ("asym", ome_asym)):
            out[f"{key}_in_ome_{tag}"] = field
            rows = []
            for ref_length, mref in FORCE_OPTS:
                fc = forces.compute_force_coeffs(im, jm, 40.0, dk, de, M[2], M[3], M[6], M[7],
                                                 M[8], M[9], field, ref_length=ref_length,
                                                 moment_ref=mref)
                rows.append([fc.cd, fc.cl, fc.cm, fc.cdp, fc.cdf, fc.clp, fc.clf, fc.cmp,
                             fc.cmf, fc.ref_length])
            out[f"{key}_out_{tag}"] = np.array(rows)
    out["force_columns"] = np.array(forces.FORCE_COLUMNS)
    velocity = load(ref_root, "velocity")
    for (im, jm) in FORCE_MESHES:
        xg, yg = mesh.generate_cylinder(im, jm, 0.5, 50.0)
        dk, de = 1.0 / (im - 1), 1.0 / (jm - 1)
        M = O.core().compute_metrics(dk, de, xg, yg)
        psi, _ = smooth_state(M[8], M[9])
        key = f"velocity_{im}x{jm}"
        for name, a in zip(("jac", "beta", "gama", "detadx", "detady"), (M[0], M[2], M[3], M[6],
                                                                          M[7])):
            out[f"{key}_in_{name}"] = a
        out[f"{key}_in_psi"] = psi
        u, v, mag = velocity.compute_velocity(im, jm, dk, de, M[0], M[2], M[3], M[6], M[7], psi,
                                              want_mag=True)
        out[f"{key}_out"] = np.stack([u, v, mag])
    rows = []
    for kw in CONFIGS:
        c = config.Config(**kw)
        rows.append([c.inv_dtau(), c.inv_2dt(), c.cos_alpha(), c.sin_alpha(),
                     float(c.ff_bc_code())] + [c.u_rot(t) for t in U_ROT_TIMES])
    out["config_scalars"] = np.array(rows)
    # the reference Config's field names and defaults, for the drop-in check
    import dataclasses
    out["config_fields"] = np.array([[f.name, repr(f.default)]
                                     for f in dataclasses.fields(config.Config)])
    dst = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst} ({os.path.getsize(dst)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VORTI2D_REFERENCE", "../reference"))
