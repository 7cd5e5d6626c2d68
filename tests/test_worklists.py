"""The GPU work lists (fmmg_worklist) rebuilt on the host from the tree and
the U/V/W/X lists (which tests/test_plan.py checks against the oracle), by the
per-node decisions of the reference evaluate(): W boxes with fewer than
|UE| x srcDOF source values and the X list of a leaf with fewer than
|DC| x trgDOF target values are summed directly (fmm3d_mpi/fmm3d_eval_mpi.cpp:1146,
1249), the others go through the UE / DC surfaces; M2L is grouped by target
parent and same-depth neighbour parent (let3d_mpi.cpp:1687-1698), and the V
lists are expanded per spectrum slot with their translation ids
(matmgnt3d_mpi.cpp:385-411 numbers the 316 offsets)."""
import numpy as np
import pytest

import fmmg

EVTR, SRCE = 4, 16


def _points(kind, n, rng):
    if kind == "uniform":
        return rng.random((n, 3))
    c = rng.uniform(0.2, 0.8, size=(6, 3))
    p = c[rng.integers(0, 6, n)] + 0.03 * rng.normal(size=(n, 3))
    return np.clip(p, 0.0, 1.0)


def _case(kt, np_, pts, kind, n, n_trg):
    rng = np.random.default_rng(kt + np_)
    src = _points(kind, n, rng)
    trg = _points("uniform", n_trg, rng) if n_trg else None
    f = fmmg.FMM3d(kt, np_=np_, pts_max=pts, device=-1)
    f.setup(src, src, trg)
    return f


def _csr_rows(ptr, idx):
    return [idx[ptr[r]:ptr[r + 1]].tolist() for r in range(len(ptr) - 1)]


@pytest.mark.parametrize("kt,np_,pts,kind,n,n_trg", [
    (111, 4, 40, "uniform", 6000, 0),
    (121, 4, 25, "clustered", 6000, 3000),
    (321, 4, 30, "clustered", 5000, 2500),
    (511, 5, 60, "uniform", 8000, 0),
    (111, 6, 12, "clustered", 4000, 4000),
])
def test_worklists_follow_the_lists(kt, np_, pts, kind, n, n_trg):
    f = _case(kt, np_, pts, kind, n, n_trg)
    rec, _, _ = f.tree()
    nn = rec.shape[0]
    depth, chd, tag, scnt, tcnt = rec[:, 0], rec[:, 5], rec[:, 6], rec[:, 7], rec[:, 8]
    leaf = chd < 0
    lsrc = leaf & (scnt > 0)
    info, st = f.info(), f.plan_stats()
    sd, td = info["src_dof"], info["trg_dof"]
    n_surf = np_ ** 3 - (np_ - 2) ** 3
    ue_size, dc_size = n_surf * st["sdm"], n_surf * st["tdm"]
    U, V, W, X = (_csr_rows(*f.lists(w)) for w in range(4))

    w_direct = lambda w: bool(lsrc[w]) and scnt[w] * sd < ue_size
    x_direct = lambda g: bool(leaf[g]) and tcnt[g] * td < dc_size
    evtr_leaves = [g for g in range(nn) if tag[g] & EVTR and leaf[g]]
    near = [U[g] + [w for w in W[g] if w_direct(w)] + (X[g] if x_direct(g) else []) for g in evtr_leaves]
    far_rows = [g for g in evtr_leaves if any(not w_direct(w) for w in W[g])]
    far = [[w for w in W[g] if not w_direct(w)] for g in far_rows]
    s2l_rows = [g for g in range(nn) if tag[g] & EVTR and not x_direct(g) and X[g]]

    rows, ptr, idx = f.worklist(0)
    assert rows.tolist() == evtr_leaves and _csr_rows(ptr, idx) == near
    rows, ptr, idx = f.worklist(1)
    assert rows.tolist() == far_rows and _csr_rows(ptr, idx) == far
    rows, ptr, idx = f.worklist(2)
    assert rows.tolist() == s2l_rows and _csr_rows(ptr, idx) == [X[g] for g in s2l_rows]
    assert f.worklist(4)[0].tolist() == [g for g in range(nn) if lsrc[g]]
    assert f.worklist(5)[0].tolist() == [g for g in evtr_leaves if depth[g] >= 2]
    # every direct or surface sum of a leaf's lists is in exactly one work list
    assert sum(len(r) for r in near) + sum(len(r) for r in far) == \
        sum(len(U[g]) + len(W[g]) + (len(X[g]) if x_direct(g) else 0) for g in evtr_leaves)

    # M2L parent pairs: same-depth non-leaf neighbours, in (dx, dy, dz) order
    at = {(int(depth[g]), *map(int, rec[g, 1:4])): g for g in range(nn)}
    want_rows, want_nbr = [], []
    for P in range(nn):
        d = int(depth[P])
        if d < 1 or leaf[P] or not any(tag[chd[P] + o] & EVTR for o in range(8)):
            continue
        q = []
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    key = (d, rec[P, 1] + dx, rec[P, 2] + dy, rec[P, 3] + dz)
                    if (dx, dy, dz) != (0, 0, 0) and key in at and not leaf[at[key]]:
                        q.append(at[key])
        if q:
            want_rows.append(P)
            want_nbr.append(q)
    rows, ptr, idx = f.worklist(3)
    assert rows.tolist() == want_rows and _csr_rows(ptr, idx) == want_nbr
    # and they give each evaluator child exactly its V list
    for P, qs in zip(want_rows, want_nbr):
        for o in range(8):
            c = chd[P] + o
            if not tag[c] & EVTR:
                continue
            got = {v for Q in qs for v in range(chd[Q], chd[Q] + 8)
                   if np.abs(rec[v, 1:4] - rec[c, 1:4]).max() > 1 and tag[v] & SRCE}
            assert got == set(V[c]), (P, c)
    # V lists only arise this way
    assert sum(len(V[g]) for g in range(nn)) == sum(
        len(V[chd[P] + o]) for P in want_rows for o in range(8) if tag[chd[P] + o] & EVTR)


def test_worklist_arguments():
    f = fmmg.FMM3d(111, np_=4, pts_max=40, device=-1)
    with pytest.raises(fmmg.FmmgError):
        f.worklist(0)  # before setup
    f.setup(np.random.default_rng(0).random((500, 3)))
    with pytest.raises(fmmg.FmmgError):
        f.worklist(8)


@pytest.mark.parametrize("kt,np_,pts,kind,n,n_trg", [
    (111, 4, 30, "clustered", 6000, 0),
    (321, 4, 25, "uniform", 5000, 3000),
])
def test_expanded_v_lists(kt, np_, pts, kind, n, n_trg):
    """Lists 6 and 7: every V entry of a target slot once, as (source slot,
    translation id of the source-minus-target offset), neighbour parent by
    neighbour parent and child by child; list 7 the same entries sorted
    stably by source slot."""
    f = _case(kt, np_, pts, kind, n, n_trg)
    rec, _, _ = f.tree()
    chd, tag = rec[:, 5], rec[:, 6]
    V = _csr_rows(*f.lists(1))
    prow, pptr, pidx = f.worklist(3)
    nbr = _csr_rows(pptr, pidx)
    tid = {}
    for a in range(-3, 4):
        for b in range(-3, 4):
            for c in range(-3, 4):
                if max(abs(a), abs(b), abs(c)) > 1:
                    tid[(a, b, c)] = len(tid)
    # slots: target children of the rows in order; source children of their
    # neighbours in first-seen order
    tnodes, tptr, tent = f.worklist(6)
    snodes, sptr, sent = f.worklist(7)
    assert tnodes.tolist() == [chd[P] + o for P in prow for o in range(8) if tag[chd[P] + o] & EVTR]
    seen = []
    for qs in nbr:
        for Q in qs:
            for v in range(chd[Q], chd[Q] + 8):
                if tag[v] & 1 and v not in seen:
                    seen.append(v)
    assert snodes.tolist() == seen
    slot_of = {int(v): s for s, v in enumerate(snodes)}
    parent_row = {int(P): r for r, P in enumerate(prow)}
    pairs = []
    for ts, t in enumerate(tnodes):
        want = []
        for Q in nbr[parent_row[int(rec[t, 4])]]:
            for v in range(chd[Q], chd[Q] + 8):
                if v in V[t]:
                    off = tuple(int(x) for x in rec[v, 1:4] - rec[t, 1:4])
                    want.append((slot_of[v], tid[off]))
        got = [tuple(e) for e in tent[tptr[ts]:tptr[ts + 1]].tolist()]
        assert got == want, t
        assert sorted(snodes[s] for s, _ in got) == sorted(V[t])
        pairs += [(s, ts, i) for s, i in got]
    assert sum(len(V[int(t)]) for t in tnodes) == len(pairs)
    inv = [(ts, i) for s, ts, i in sorted(pairs, key=lambda e: e[0])]  # stable
    assert [tuple(e) for e in sent.tolist()] == inv
    assert sptr.tolist() == np.concatenate([[0], np.cumsum(np.bincount([p[0] for p in pairs],
                                                                        minlength=len(snodes)))]).tolist()


def test_lazy_lists_follow_each_setup():
    """The expanded V lists are formed on first use after each setup: a
    handle that formed them for one point set and is set up again on another
    returns the new set's lists, the same as a fresh handle's, and the
    setup's last phase (the adjoint's lists, formed on first use too) is empty."""
    rng = np.random.default_rng(41)
    a_pts, b_pts = _points("clustered", 5000, rng), _points("uniform", 7000, rng)
    f = fmmg.FMM3d(111, np_=4, pts_max=30, device=-1)
    f.setup(a_pts)
    first = [x.copy() for x in f.worklist(6)]
    f.setup(b_pts)
    assert f.setup_times()["adjoint_lists"] < 1.0  # ms: only the lazily formed lists are reset
    g = fmmg.FMM3d(111, np_=4, pts_max=30, device=-1)
    g.setup(b_pts)
    for which in (6, 7):
        for x, y in zip(f.worklist(which), g.worklist(which)):
            assert np.array_equal(x, y)
    assert not all(np.array_equal(x, y) for x, y in zip(first, f.worklist(6)))
