"""Inputs shared by the CPU and GPU tests."""
import numpy as np


def smooth_state(x, y):
    """Seam-consistent analytic state of the reference's local-assembly test
    (tests/test_assemble_local.py:23-30)."""
    r = np.sqrt(x ** 2 + y ** 2)
    psi = np.sin(0.3 * x) * np.cos(0.2 * y) / (1.0 + 0.01 * r)
    ome = np.cos(0.25 * x) * np.sin(0.15 * y) * np.exp(-0.02 * r)
    return psi, ome, 0.9 * ome, 0.8 * ome


def local_layout(imax, jmax):
    """1-rank periodic DMDA layout (ni = imax-1 columns, one ghost column on
    each side, dof=2 node-interleaved natural ordering), as
    vorti2d/domain.py:41-63 sets it up on one rank."""
    ni = imax - 1
    gxs, gxm = -1, ni + 2
    il0, il1 = 2, gxm - 1
    gc = (gxs + np.arange(gxm)) % ni
    lg = np.empty(2 * gxm * jmax, dtype=np.intc)
    for j in range(jmax):
        for il in range(gxm):
            K = j * gxm + il
            lg[2 * K] = (j * ni + gc[il]) * 2
            lg[2 * K + 1] = (j * ni + gc[il]) * 2 + 1
    return ni, gxs, gxm, il0, il1, gc, lg


def to_local(field, imax, jmax, gxm, gc):
    """Global pointer-order field -> ghosted local block (gxm x jmax)."""
    g2 = field.reshape(jmax, imax)[:, :imax - 1]
    return np.ascontiguousarray(g2[:, gc].ravel())
