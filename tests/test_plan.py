"""CPU checks of the library's host plan (tree, lists, operators) against the oracle.

The tree and the U/V/W/X lists are integer work: they must match the oracle's
restatement of fmm3d_mpi/let3d_mpi.cpp:611-726, 1209-1768 exactly (node sets,
point binning, list membership), after mapping the two node numberings by
(depth, path).  Operators are compared numerically.  Uses host-only handles
(device=-1), so no GPU is touched.
"""
import numpy as np
import pytest

import fmmg
import oracle as O


def _clustered(rng, n):
    a = rng.random((n // 2, 3))
    c = rng.uniform(0.2, 0.8, size=(4, 3))
    b = c[rng.integers(0, 4, n - n // 2)] + 0.03 * rng.normal(size=(n - n // 2, 3))
    return np.clip(np.concatenate([a, b]), 0.0, 1.0)


def _pair(kt, np_, pts, src, trg, nrm=None):
    lib = fmmg.FMM3d(kt, np_=np_, pts_max=pts, device=-1)
    lib.setup(src, nrm if nrm is not None else src, trg)
    orc = O.Oracle(kt, np_=np_, pts_max=pts)
    orc.setup(src, nrm if nrm is not None else src, trg)
    return lib, orc


def _keymaps(lib, orc):
    rec, _, _ = lib.tree()
    nd = orc.nodes()
    lk = {(r[0], r[1], r[2], r[3]): i for i, r in enumerate(rec)}
    ok = {(r[0], r[1], r[2], r[3]): i for i, r in enumerate(nd)}
    return rec, nd, lk, ok


# the 150,000-point case has top-level nodes above the size at which the
# library partitions a node's points with all threads (sources and targets)
@pytest.mark.parametrize("dist,pts,sep,n", [("uniform", 40, False, 6000), ("clustered", 25, False, 6000),
                                            ("clustered", 30, True, 6000), ("uniform", 60, True, 150000)])
def test_tree_and_lists_identical_to_oracle(dist, pts, sep, n):
    rng = np.random.default_rng(5)
    src = rng.random((n, 3)) if dist == "uniform" else _clustered(rng, n)
    trg = rng.random((2500 if n <= 6000 else n // 2, 3)) if sep else src
    lib, orc = _pair(111, 4, pts, src, trg)
    rec, nd, lk, ok = _keymaps(lib, orc)
    assert set(lk) == set(ok)
    l2o = np.array([ok[(r[0], r[1], r[2], r[3])] for r in rec])
    # per node: source / target counts and evaluator / contributor / has-sources tags
    np.testing.assert_array_equal(rec[:, 7], nd[l2o, 7])
    np.testing.assert_array_equal(rec[:, 8], nd[l2o, 8])
    for bit in (1, 4, 16):
        np.testing.assert_array_equal(rec[:, 6] & bit, nd[l2o, 6] & bit)
    # every leaf holds the same sources in the same (input) order; the library
    # lays leaves out in Morton order, the oracle in the reference's
    # node-creation order (let3d_mpi.cpp:611-726, 1436-1462)
    _, lps, lpt = lib.tree()
    ops, _ = orc.perms()
    leaves = [i for i in range(len(rec)) if rec[i, 5] < 0 and rec[i, 7] > 0]
    D = int(rec[:, 0].max())

    def morton(i):
        d, x, y, z = (int(v) for v in rec[i, :4])
        x, y, z = x << (D - d), y << (D - d), z << (D - d)
        code = 0
        for b in range(D - 1, -1, -1):
            code = (code << 3) | (((x >> b) & 1) << 2) | (((y >> b) & 1) << 1) | ((z >> b) & 1)
        return code

    beg = 0
    for i in sorted(leaves, key=morton):
        cnt = rec[i, 7]
        ob = nd[l2o[i], 9]
        np.testing.assert_array_equal(lps[beg:beg + cnt], ops[ob:ob + cnt])
        beg += cnt
    assert beg == len(src)
    np.testing.assert_array_equal(np.sort(lpt), np.arange(len(trg)))
    for which in range(4):
        lp, li = lib.lists(which)
        op, oi = orc.lists(which)
        for a in range(len(rec)):
            mine = sorted(l2o[li[lp[a]:lp[a + 1]]])
            theirs = sorted(oi[op[l2o[a]]:op[l2o[a] + 1]])
            assert mine == theirs, (which, a)


def test_grouped_vlist_equals_reference_vlist():
    # the GPU M2L groups V-lists by (parent, neighbour parent); the implied
    # lists must equal the reference-form V-lists of let3d_mpi.cpp:1687-1698
    rng = np.random.default_rng(9)
    src = _clustered(rng, 8000)
    lib = fmmg.FMM3d(111, np_=4, pts_max=20, device=-1)
    lib.setup(src)
    rec, _, _ = lib.tree()
    depth, path, chd = rec[:, 0], rec[:, 1:4], rec[:, 5]
    key = {(d, x, y, z): i for i, (d, x, y, z) in enumerate(rec[:, :4])}
    vp, vi = lib.lists(1)
    for c in range(len(rec)):
        if c == 0 or not (rec[c, 6] & 4):
            continue
        P = rec[c, 4]
        implied = []
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    if (dx, dy, dz) == (0, 0, 0):
                        continue
                    q = key.get((depth[P], path[P, 0] + dx, path[P, 1] + dy, path[P, 2] + dz))
                    if q is None or chd[q] < 0:
                        continue
                    for o in range(8):
                        v = chd[q] + o
                        if np.abs(path[v] - path[c]).max() >= 2 and (rec[v, 6] & 16):
                            implied.append(v)
        assert sorted(implied) == sorted(vi[vp[c]:vp[c + 1]].tolist()), c


@pytest.mark.parametrize("kt,np_", [(111, 4), (111, 6), (321, 4), (511, 4)])
def test_operators_match_oracle(kt, np_):
    rng = np.random.default_rng(1)
    src = rng.random((500, 3))
    lib, orc = _pair(kt, np_, 100, src, src, nrm=src)
    eps = 0.1 ** (np_ + 1)
    # M2M / L2L kernel matrices and the translation spectra are plain kernel
    # evaluations (+ a DFT): agree to rounding
    for which, idxs in ((1, range(8)), (3, range(8)), (4, (0, 57, 200, 315))):
        for i in idxs:
            a, b = lib.operator(which, i), orc.operator(which, i)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max())
    # pseudo-inverses from two SVD codes agree to ~eps_mach / cutoff
    for which in (0, 2):
        a, b = lib.operator(which), orc.operator(which)
        np.testing.assert_allclose(a, b, rtol=0, atol=100 * 1e-16 / eps * np.abs(b).max())


def test_library_exports_every_declared_symbol():
    import ctypes
    import os
    import re
    hdr = open(os.path.join(os.path.dirname(fmmg.__file__), "..", "include", "fmmg.h")).read()
    names = set(re.findall(r"\b(fmmg_[a-z_]+)\s*\(", hdr))
    assert names, "no declarations found"
    L = ctypes.CDLL(fmmg.LIB_PATH)
    for n in names:
        assert hasattr(L, n), n
    assert names == set(fmmg.SIGNATURES)


def test_invalid_arguments_are_reported_not_fatal():
    with pytest.raises(fmmg.FmmgError) as e:
        fmmg.FMM3d(999, device=-1)
    assert e.value.status == fmmg.FMMG_NOT_SUPPORTED
    with pytest.raises(fmmg.FmmgError) as e:
        fmmg.FMM3d(111, np_=2, device=-1)
    assert e.value.status == fmmg.FMMG_NOT_SUPPORTED
    with pytest.raises(fmmg.FmmgError) as e:
        fmmg.FMM3d(111, pts_max=0, device=-1)
    assert e.value.status == fmmg.FMMG_INVALID_ARG
    f = fmmg.FMM3d(111, np_=4, device=-1)
    bad = np.random.default_rng(0).random((100, 3))
    bad[7, 1] = np.nan
    with pytest.raises(fmmg.FmmgError) as e:
        f.setup(bad)
    assert e.value.status == fmmg.FMMG_INVALID_ARG
    bad[7, 1] = 1.5  # outside the root box
    with pytest.raises(fmmg.FmmgError) as e:
        f.setup(bad)
    assert e.value.status == fmmg.FMMG_INVALID_ARG
    with pytest.raises(fmmg.FmmgError) as e:  # double layer without normals
        g = fmmg.FMM3d(121, np_=4, device=-1)
        g.setup(np.random.default_rng(0).random((10, 3)))
    assert e.value.status == fmmg.FMMG_INVALID_ARG
    with pytest.raises(fmmg.FmmgError) as e:  # evaluate before setup
        fmmg.FMM3d(111, np_=4, device=-1).evaluate(np.zeros(0))
    assert e.value.status in (fmmg.FMMG_STATE, fmmg.FMMG_INVALID_ARG)


def test_degenerate_inputs_build_a_plan():
    f = fmmg.FMM3d(111, np_=4, pts_max=10, device=-1)
    f.setup(np.array([[0.3, 0.3, 0.3]]))  # one point: the root is still split
    info = f.info()
    assert info["nodes"] == 9 and info["leaves"] == 8
    p = np.full((50, 3), 0.25)  # coincident points: split down to max_level
    g = fmmg.FMM3d(111, np_=4, pts_max=10, max_level=5, device=-1)
    g.setup(p)
    assert g.info()["max_depth"] == 5
    edge = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.5, 0.5, 0.5], [1.0, 0.0, 0.5]])
    h = fmmg.FMM3d(111, np_=4, pts_max=1, device=-1)
    h.setup(edge)
    _, ps, _ = h.tree()
    assert sorted(ps.tolist()) == [0, 1, 2, 3]


@pytest.mark.parametrize("np_", [4, 5, 6])
def test_plan_stats_of_the_mixed_form(np_):
    """The mixed form's own work figures: its spectra live on the
    (2np-1)^3 grid (r2c half spectrum, no Nyquist term), and folding the
    upward C2E into M2M for parents needs fewer upward FLOPs than the
    reference's M2M + C2E."""
    rng = np.random.default_rng(31 + np_)
    lib = fmmg.FMM3d(111, np_=np_, pts_max=20, device=-1)
    lib.setup(_clustered(rng, 6000))
    s = lib.plan_stats()
    n, m = 2 * np_, 2 * np_ - 1
    assert s["n_eff"] == n * n * (n // 2 + 1)
    assert s["n_eff_mixed"] == m * m * (m // 2 + 1) == m * m * np_
    assert 0 < s["up_gemm_flops_mixed"] < s["up_gemm_flops"]
    assert s["dn_gemm_flops_mixed"] > 0
    w64, w32 = lib.algorithmic_work(k=8, precision="fp64"), lib.algorithmic_work(k=8, precision="fp32")
    assert w32["m2l_had"]["flops"] * s["n_eff"] == w64["m2l_had"]["flops"] * s["n_eff_mixed"]
