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


def flow_plan(v2d, imax, jmax, ip, ix, leaf=64):
    from vorti2d_b200 import _lib
    info = np.zeros(4, dtype=np.intc)
    code = _lib.lib().v2d_lu_flow_plan(imax, jmax, _lib.iptr(ip), _lib.iptr(ix), leaf,
                                       _lib.iptr(info), None, 0, None, 0)
    assert code == 0, v2d._lib.last_error()
    items = np.zeros(4 * max(int(info[1]), 1), dtype=np.intc)
    parent = np.zeros(max(int(info[3]), 1), dtype=np.intc)
    code = _lib.lib().v2d_lu_flow_plan(imax, jmax, _lib.iptr(ip), _lib.iptr(ix), leaf,
                                       _lib.iptr(info), _lib.iptr(items), int(info[1]),
                                       _lib.iptr(parent), int(info[3]))
    assert code == 0, v2d._lib.last_error()
    return info, items[:4 * int(info[1])].reshape(-1, 4), parent[:int(info[3])]


FZ, FU, BY, BX, BXROOT = range(5)


def _wait_ctr(kind, q, parent, nf):
    # the counter each kind waits on (4 per front: z, children's contribution, y, x)
    return {FZ: nf + q, FU: q, BY: 3 * nf + parent[q] if parent[q] >= 0 else -1,
            BX: 2 * nf + q, BXROOT: q}[kind]


def _done_ctr(kind, q, parent, nf):
    return {FZ: q, FU: nf + parent[q] if parent[q] >= 0 else -1, BY: 2 * nf + q,
            BX: 3 * nf + q, BXROOT: 3 * nf + q}[kind]


def _producers(items, parent):
    """What each item reads, from the algorithm alone (not from the
    counters): z rows need every contribution chunk of the front's children;
    contribution rows every z chunk of the front; backward y rows the
    front's z and the x chunks of every ancestor (its contribution variables
    are pivots of ancestors); x rows the front's z and y chunks."""
    by_kind = {}
    for k, (kind, q, c, t) in enumerate(items):
        by_kind.setdefault((kind, q), []).append(k)
    kids = {}
    for k, (kind, q, c, t) in enumerate(items):
        if kind == FU:
            kids.setdefault(parent[q], set()).add(q)

    def xs(a):
        return by_kind.get((BX, a), []) + by_kind.get((BXROOT, a), [])

    prod = []
    for kind, q, c, t in items:
        if kind == FZ:
            p = [k for ch in kids.get(q, ()) for k in by_kind[(FU, ch)]]
        elif kind == FU:
            p = by_kind[(FZ, q)]
        elif kind == BY:
            p = list(by_kind[(FZ, q)])
            a = parent[q]
            while a >= 0:
                p += xs(a)
                a = parent[a]
        else:
            p = by_kind[(FZ, q)] + by_kind.get((BY, q), [])
        prod.append(p)
    return prod


def _simulate(items, parent, nf, ctas, rng):
    """The kernel's schedule: CTAs take items in ticket order, wait on one
    counter, finish after a random time, count the item.  Returns the finish
    order; fails on a deadlock or on an item starting before what it reads."""
    n = len(items)
    ctr = np.zeros(4 * nf, dtype=np.int64)
    prod = _producers(items, parent)
    done = np.zeros(n, dtype=bool)
    ticket = 0
    held = {}            # cta -> [item, finish time or None while waiting]
    now, order = 0.0, []
    for cta in range(ctas):
        if ticket < n:
            held[cta] = [ticket, None]
            ticket += 1
    while held:
        progressed = False
        for cta, slot in list(held.items()):
            k = slot[0]
            kind, q, c, t = items[k]
            if slot[1] is None:
                w = _wait_ctr(kind, q, parent, nf)
                if t <= 0 or ctr[w] >= t:
                    assert all(done[p] for p in prod[k]), (k, items[k])
                    slot[1] = now + rng.uniform(0.5, 2.0)
                    progressed = True
        running = [(s[1], cta) for cta, s in held.items() if s[1] is not None]
        assert running or progressed, "deadlock"
        if not running:
            continue
        tfin, cta = min(running)
        now = tfin
        k = held[cta][0]
        kind, q, c, t = items[k]
        d = _done_ctr(kind, q, parent, nf)
        if d >= 0:
            ctr[d] += 1
        done[k] = True
        order.append(k)
        if ticket < n:
            held[cta] = [ticket, None]
            ticket += 1
        else:
            del held[cta]
    assert done.all()
    return order


@pytest.mark.parametrize("imax,jmax,leaf", [(5, 4, 64), (9, 7, 4), (24, 13, 16), (33, 21, 16),
                                            (65, 49, 64), (129, 129, 64), (181, 181, 64),
                                            (257, 129, 64)])
def test_flow_plan_order_is_safe(v2d, oracle_mod, imax, jmax, leaf):
    """The dataflow solve's work items: validated by the plan, every front
    above the one-CTA-per-front levels appears with the chunk counts of its
    rows, and a simulated schedule (1 to 300 CTAs, random item times) never
    deadlocks and never starts an item before the items it reads."""
    ip, ix = pattern(oracle_mod, imax, jmax, 1)
    info, items, parent = flow_plan(v2d, imax, jmax, ip, ix, leaf)
    L0, nflow, valid, nf = (int(v) for v in info)
    assert valid == 1 and nflow == len(items) > 0
    kinds = set(items[:, 0].tolist())
    assert {FZ, FU, BX} <= kinds and BXROOT in kinds
    # forward items precede backward ones
    fwd = np.isin(items[:, 0], [FZ, FU])
    assert fwd[:fwd.sum()].all()
    rng = np.random.default_rng(imax * 7 + jmax)
    for ctas in (1, 2, 5, 37, 300):
        order = _simulate(items, parent, nf, ctas, rng)
        assert len(order) == nflow


def test_flow_plan_181_levels(v2d, oracle_mod):
    """181x181, 64-node leaves: levels 0-3 (512, 256, 128, 64 fronts) keep
    the one-CTA-per-front launches; the other 65 fronts (levels 4-10) form
    the dataflow, the root last."""
    ip, ix = pattern(oracle_mod, 181, 181, 1)
    info, items, parent = flow_plan(v2d, 181, 181, ip, ix)
    assert int(info[0]) == 4 and int(info[3]) == 1025
    fronts = sorted(set(items[:, 1].tolist()))
    assert fronts == list(range(960, 1025))
    assert parent[1024] == -1 and (parent[960:1024] >= 960).all()


def test_plan_rejects_malformed_csr(v2d, oracle_mod):
    """Column indices outside [0, n) and decreasing row pointers are argument
    errors, found before any index is used."""
    from vorti2d_b200 import _lib
    ip, ix = pattern(oracle_mod, 33, 21, 1)
    bad = ix.copy()
    bad[len(bad) // 2] = 2 * 33 * 21
    code, _ = plan_info(v2d, 33, 21, ip, bad)
    assert code == _lib.V2D_EARG and b"outside" in _lib.lib().v2d_last_error()
    bad = ix.copy()
    bad[3] = -1
    code, _ = plan_info(v2d, 33, 21, ip, bad)
    assert code == _lib.V2D_EARG
    bip = ip.copy()
    bip[10] = bip[12] + 1
    code, _ = plan_info(v2d, 33, 21, bip, ix)
    assert code == _lib.V2D_EARG and b"decreases" in _lib.lib().v2d_last_error()
