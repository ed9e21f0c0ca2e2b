"""Host-side symbolic analysis of the multifrontal LU preconditioner
(v2d_lu_plan_info: no device work) over grid shapes, far-field BCs and leaf
sizes.  The plan builder checks that every index the factorization and solve
kernels dereference stays inside its buffer and that no separator couples
across sibling subtrees; these tests exercise that on the canonical CSR
patterns the oracle's assembly produces."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from cases import smooth_state


def pattern(O, imax, jmax, ff_bc, adeg=0.0):
    xg, yg = O.generate_cylinder(imax, jmax)
    dk, de = 1 / (imax - 1), 1 / (jmax - 1)
    M = O.core().compute_metrics(dk, de, xg, yg)
    N = imax * jmax
    ci, cj, cv, nnz, _ = O.core().assemble_coo(
        imax, jmax, 80.0, 0.0, 2.5, 0.3, dk, de, *M, *smooth_state(M[8], M[9]), 0, 2 * N,
        26 * N, ff_bc, np.cos(np.radians(adeg)), np.sin(np.radians(adeg)))
    A = sp.csr_matrix((cv[:nnz], (ci[:nnz], cj[:nnz])), shape=(2 * N, 2 * N))
    return A.indptr.astype(np.intc), A.indices.astype(np.intc)


def plan_info(v2d, imax, jmax, ip, ix, leaf=64):
    from vorti2d_b200 import _lib
    out = (ctypes.c_longlong * 8)()
    code = _lib.lib().v2d_lu_plan_info(imax, jmax, _lib.iptr(ip), _lib.iptr(ix), leaf, out)
    return code, list(out)


@pytest.mark.parametrize("imax,jmax", [(5, 4), (6, 4), (9, 7), (24, 13), (33, 21), (64, 48),
                                       (129, 129), (181, 181), (257, 129), (257, 193)])
@pytest.mark.parametrize("ff_bc", [0, 1, 2])
def test_plan_builds_and_checks_indices(v2d, oracle_mod, imax, jmax, ff_bc):
    ip, ix = pattern(oracle_mod, imax, jmax, ff_bc, adeg=8.0 if ff_bc == 2 else 0.0)
    code, (nfront, nlevel, maxS, maxf, ftot, flops, vtot, utot) = plan_info(v2d, imax, jmax,
                                                                            ip, ix)
    assert code == 0, v2d._lib.last_error()
    assert nfront >= 1 and nlevel >= 1
    # the root separator: the middle circumferential row (2 imax unknowns), or
    # on grids with fewer than 8 rows the seam columns plus the middle column
    assert maxS >= (2 * imax if jmax >= 8 else 3 * 2 * jmax)
    assert maxf >= maxS and ftot >= maxf * maxf
    # the solve's shared vectors (FP64) fit in shared memory
    assert (maxf + maxS) * 8 <= 227 * 1024


@pytest.mark.parametrize("leaf", [4, 16, 64, 256])
def test_plan_leaf_sizes(v2d, oracle_mod, leaf):
    ip, ix = pattern(oracle_mod, 65, 49, 1)
    code, info = plan_info(v2d, 65, 49, ip, ix, leaf)
    assert code == 0, v2d._lib.last_error()


def test_plan_181_shape(v2d, oracle_mod):
    """181x181 with 64-node leaves: 1025 fronts over 11 levels; the root is
    the middle circumferential row (362 unknowns), the two annulus fronts
    hold the seam half-columns; largest front 902 unknowns, about 7.3 GFLOP
    per factorization."""
    ip, ix = pattern(oracle_mod, 181, 181, 1)
    code, (nfront, nlevel, maxS, maxf, ftot, flops, vtot, utot) = plan_info(v2d, 181, 181, ip, ix)
    assert code == 0
    assert (nfront, nlevel, maxS, maxf) == (1025, 11, 362, 902)
    assert 7.0e9 < flops < 7.5e9


def test_plan_rejects_bad_input(v2d, oracle_mod):
    """Argument checks that run before any array is read."""
    from vorti2d_b200 import _lib
    ip, ix = pattern(oracle_mod, 9, 7, 0)
    code, _ = plan_info(v2d, 4, 7, ip, ix)      # grid too small for a separator tree
    assert code == _lib.V2D_EARG
    out = (ctypes.c_longlong * 8)()
    assert _lib.lib().v2d_lu_plan_info(9, 7, None, None, 64, out) == _lib.V2D_EARG
