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


def solve_plan(v2d, imax, jmax, ip, ix, leaf=64):
    """The solve's work items (12 ints each) and (S, f, parent) per front."""
    from vorti2d_b200 import _lib
    info = np.zeros(4, dtype=np.intc)
    code = _lib.lib().v2d_lu_solve_plan(imax, jmax, _lib.iptr(ip), _lib.iptr(ix), leaf,
                                        _lib.iptr(info), None, 0, None, 0)
    assert code == 0, v2d._lib.last_error()
    ni, nc, nf, nl = (int(v) for v in info)
    items = np.zeros(12 * max(ni, 1), dtype=np.intc)
    fronts = np.zeros(3 * max(nf, 1), dtype=np.intc)
    code = _lib.lib().v2d_lu_solve_plan(imax, jmax, _lib.iptr(ip), _lib.iptr(ix), leaf,
                                        _lib.iptr(info), _lib.iptr(items), ni,
                                        _lib.iptr(fronts), nf)
    assert code == 0, v2d._lib.last_error()
    return (ni, nc, nf, nl), items[:12 * ni].reshape(-1, 12), fronts[:3 * nf].reshape(-1, 3)


FWD, BWD, FWD_GATHER, BWD_GATHER = 0, 1, 2, 3


def _producers(items, fronts):
    """What each item reads (or overwrites), from the algorithm alone (not
    from the counters): a forward item gathers its children's contribution
    rows, or reads what its front's forward gather item gathered; a backward
    item multiplies its front's z rows and the x of every ancestor (the
    front's contribution variables are pivots of ancestors), or the x its
    front's backward gather item collected; a backward gather item reads the
    ancestors' x and overwrites the w part that the front's forward
    contribution rows read."""
    S, f, parent = fronts[:, 0], fronts[:, 1], fronts[:, 2]
    kids = {}
    for q, pa in enumerate(parent):
        if pa >= 0:
            kids.setdefault(int(pa), []).append(q)
    fwd_cb, fwd_z, bwd, fg, bg = {}, {}, {}, {}, {}
    for k, it in enumerate(items):
        kind, q, rb, re = (int(v) for v in it[:4])
        if kind == FWD:
            if re > S[q]:
                fwd_cb.setdefault(q, []).append(k)
            if rb < S[q]:
                fwd_z.setdefault(q, []).append(k)
        elif kind == BWD:
            bwd.setdefault(q, []).append(k)
        elif kind == FWD_GATHER:
            fg.setdefault(q, []).append(k)
        else:
            bg.setdefault(q, []).append(k)

    def ancestors_x(q):
        p, a = [], parent[q]
        while a >= 0:
            p += bwd.get(int(a), [])
            a = parent[a]
        return p

    prod = []
    for it in items:
        kind, q, gathered = int(it[0]), int(it[1]), int(it[11])
        if kind == FWD:
            prod.append(list(fg[q]) if gathered
                        else [k for c in kids.get(q, ()) for k in fwd_cb.get(c, [])])
        elif kind == FWD_GATHER:
            prod.append([k for c in kids.get(q, ()) for k in fwd_cb.get(c, [])])
        elif kind == BWD:
            prod.append(list(fwd_z.get(q, [])) + (list(bg[q]) if gathered else ancestors_x(q)))
        else:
            prod.append(ancestors_x(q) + list(fwd_cb.get(q, [])))
    return prod


def _simulate(items, fronts, nc, ctas, rng):
    """The kernel's schedule: CTAs take items in ticket order, wait until both
    of the item's counters reach their targets, finish after a random time
    and add one to the item's done counters.  Fails on a deadlock or on an
    item starting before what it reads; returns the finish order."""
    n = len(items)
    ctr = np.zeros(nc, dtype=np.int64)
    prod = _producers(items, fronts)
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
            it = items[k]
            if slot[1] is None:
                ready = all(c < 0 or t <= 0 or ctr[c] >= t for c, t in ((it[4], it[5]),
                                                                         (it[6], it[7])))
                if ready:
                    assert all(done[p] for p in prod[k]), (k, it)
                    slot[1] = now + rng.uniform(0.5, 2.0)
                    progressed = True
        running = [(s[1], cta) for cta, s in held.items() if s[1] is not None]
        assert running or progressed, "deadlock"
        if not running:
            continue
        tfin, cta = min(running)
        now = tfin
        k = held[cta][0]
        for d in items[k][8:10]:
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
def test_solve_plan_order_is_safe(v2d, oracle_mod, imax, jmax, leaf):
    """The solve's work items: every front's forward rows [0, f) and backward
    rows [0, S) are covered exactly once, forward items precede backward
    ones, and a simulated dataflow schedule (1 to 300 CTAs, random item
    times) never deadlocks and never starts an item before the items it
    reads."""
    ip, ix = pattern(oracle_mod, imax, jmax, 1)
    (ni, nc, nf, nl), items, fronts = solve_plan(v2d, imax, jmax, ip, ix, leaf)
    assert ni == len(items) > 0 and nc == 5 * nf
    assert (items[:, 0] <= BWD).all()   # the default split has no gather items
    S, f = fronts[:, 0], fronts[:, 1]
    cover = {}
    for it in items:
        cover.setdefault((int(it[0]), int(it[1])), []).append((int(it[2]), int(it[3])))
    for q in range(nf):
        for kind, end in ((FWD, f[q]), (BWD, S[q])):
            rows = sorted(cover[(kind, q)])
            assert rows[0][0] == 0 and rows[-1][1] == end
            assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
    fwd = items[:, 0] == FWD
    assert fwd[:fwd.sum()].all()
    rng = np.random.default_rng(imax * 7 + jmax)
    for ctas in (1, 2, 5, 37, 300):
        order = _simulate(items, fronts, nc, ctas, rng)
        assert len(order) == ni


def solve_plan_split(v2d, imax, jmax, ip, ix, rows, leaf=64):
    """solve_plan with an explicit rows-per-item entry per level."""
    from vorti2d_b200 import _lib
    r = np.ascontiguousarray(rows, dtype=np.intc)
    info = np.zeros(4, dtype=np.intc)
    code = _lib.lib().v2d_lu_solve_plan_split(imax, jmax, _lib.iptr(ip), _lib.iptr(ix), leaf,
                                              _lib.iptr(r), r.size, _lib.iptr(info), None, 0,
                                              None, 0)
    assert code == 0, v2d._lib.last_error()
    ni, nc, nf, nl = (int(v) for v in info)
    items = np.zeros(12 * ni, dtype=np.intc)
    fronts = np.zeros(3 * nf, dtype=np.intc)
    code = _lib.lib().v2d_lu_solve_plan_split(imax, jmax, _lib.iptr(ip), _lib.iptr(ix), leaf,
                                              _lib.iptr(r), r.size, _lib.iptr(info),
                                              _lib.iptr(items), ni, _lib.iptr(fronts), nf)
    assert code == 0, v2d._lib.last_error()
    return (ni, nc, nf, nl), items.reshape(-1, 12), fronts.reshape(-1, 3)


@pytest.mark.parametrize("imax,jmax,leaf,split", [
    (33, 21, 16, "neg8"), (65, 49, 64, "neg8"), (181, 181, 64, "mixed"),
    (257, 129, 64, "neg32")])
def test_gathered_split_order_is_safe(v2d, oracle_mod, imax, jmax, leaf, split):
    """Negative rows-per-item entries: a front split into several items gets
    one forward gather item (before its level's row items) and, if it has
    struct variables, one backward gather item; every front's rows are still
    covered exactly once, the items of split fronts carry the gathered flag,
    and the simulated dataflow schedule never deadlocks nor starts an item
    before what it reads or overwrites."""
    ip, ix = pattern(oracle_mod, imax, jmax, 1)
    (_, _, _, nl), _, _ = solve_plan(v2d, imax, jmax, ip, ix, leaf)
    rows = {"neg8": [-8] * nl, "neg32": [-32] * nl,
            "mixed": [0 if L < 3 else (-16 if L % 2 else 8) for L in range(nl)]}[split]
    (ni, nc, nf, nl2), items, fronts = solve_plan_split(v2d, imax, jmax, ip, ix, rows, leaf)
    assert nl2 == nl and ni == len(items) and nc == 5 * nf
    S, f = fronts[:, 0], fronts[:, 1]
    lvl = {}
    for it in items:
        lvl[int(it[1])] = int(it[10])
    n_fg = n_bg = 0
    for q in range(nf):
        R = rows[lvl[q]]
        split_f = R < 0 and f[q] > -R
        split_b = R < 0 and S[q] > -R and f[q] > S[q]
        mine = items[items[:, 1] == q]
        assert (mine[:, 0] == FWD_GATHER).sum() == int(split_f)
        assert (mine[:, 0] == BWD_GATHER).sum() == int(split_b)
        n_fg += int(split_f)
        n_bg += int(split_b)
        for kind, end, flag in ((FWD, f[q], split_f), (BWD, S[q], split_b)):
            rr = sorted((int(a), int(b)) for a, b in mine[mine[:, 0] == kind][:, 2:4])
            assert rr[0][0] == 0 and rr[-1][1] == end
            assert all(a[1] == b[0] for a, b in zip(rr, rr[1:]))
            assert (mine[mine[:, 0] == kind][:, 11] == int(flag)).all()
    assert n_fg > 0
    rng = np.random.default_rng(imax + jmax)
    for ctas in (1, 3, 37, 300):
        assert len(_simulate(items, fronts, nc, ctas, rng)) == ni


def test_solve_plan_181_items(v2d, oracle_mod):
    """181x181, 64-node leaves: the default split aims at about 600 items per
    level -- R rows per item, R the level's rows over 600 rounded down to a
    power of two in [8, 256], whole fronts where no front of the level has
    more than R rows; the root (362 pivots, no contribution rows) is the last
    forward front and the first backward one."""
    ip, ix = pattern(oracle_mod, 181, 181, 1)
    (ni, nc, nf, nl), items, fronts = solve_plan(v2d, 181, 181, ip, ix)
    assert (nf, nl) == (1025, 11)
    for L in range(nl):
        it = items[items[:, 10] == L]
        qs = np.unique(it[:, 1])
        rows = int(fronts[qs, 1].sum())
        R = 8
        while R < 256 and 2 * R * 600 <= rows:
            R *= 2
        span = it[:, 3] - it[:, 2]
        if fronts[qs, 1].max() <= R:
            assert (it[:, 2] == 0).all()
            assert (it[:, 3] == np.where(it[:, 0] == FWD, fronts[it[:, 1], 1],
                                         fronts[it[:, 1], 0])).all()
        else:
            assert span.max() == R and (span > 0).all()
            # every chunk but a front's last is full
            last = it[:, 3] == np.where(it[:, 0] == FWD, fronts[it[:, 1], 1],
                                        fronts[it[:, 1], 0])
            assert (span[~last] == R).all()
    fwd = items[items[:, 0] == FWD]
    bwd = items[items[:, 0] == BWD]
    assert fwd[-1, 1] == 1024 and bwd[0, 1] == 1024 and fronts[1024, 2] == -1
    assert fronts[1024, 0] == fronts[1024, 1] == 362


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
