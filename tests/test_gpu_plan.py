"""The plan built on the GPU (tree_gpu.cu: octree and target binning;
lists_gpu.cu: U/V/W/X lists) against the host build (plan.cpp, the
restatement of let3d_mpi.cpp:611-726, 1230-1285, 1470-1538, 1637-1768): the
same nodes, permutations, ranges, lists and work lists, bit for bit, on the
workloads' point sets and the edge cases the tree has (coincident points that
hit max_level, points on box faces, separate targets, a single point)."""
import numpy as np
import pytest

import fmmg
import workloads as W

pytestmark = pytest.mark.gpu


def _plans(src, trg=None, **kw):
    a = fmmg.FMM3d(111, np_=4, device=0, **kw)
    b = fmmg.FMM3d(111, np_=4, device=0, **kw)
    b.set_tree_device(False)
    a.setup(src, None, trg)
    b.setup(src, None, trg)
    return a, b


def _same(a, b):
    ra, psa, pta = a.tree()
    rb, psb, ptb = b.tree()
    assert ra.shape == rb.shape
    assert np.array_equal(ra, rb)
    assert np.array_equal(psa, psb)
    assert np.array_equal(pta, ptb)
    for which in range(4):
        pa, ia = a.lists(which)
        pb, ib = b.lists(which)
        assert np.array_equal(pa, pb) and np.array_equal(ia, ib)
    for which in range(8):
        for x, y in zip(a.worklist(which), b.worklist(which)):
            assert (x is None and y is None) or np.array_equal(x, y)


def _edge_sets():
    rng = np.random.default_rng(11)
    out = {}
    out["sphere_clusters_200k"] = (W.sphere_clusters(200000, rng), None, dict(pts_max=64))
    out["uniform_100k_targets_apart"] = (W.uniform(100000, rng), W.uniform(70000, rng), dict(pts_max=40))
    pts = rng.random((3000, 3))
    pts[:500] = 0.25  # coincident points: splits stop at max_level
    out["coincident_max_level"] = (pts, None, dict(pts_max=30, max_level=9))
    g = np.linspace(0.0, 1.0, 17)
    grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)  # points on box faces
    out["grid_on_faces"] = (grid, None, dict(pts_max=8))
    out["single_point"] = (np.array([[0.3, 0.6, 0.9]]), None, dict(pts_max=1))
    return out


@pytest.mark.parametrize("name", list(_edge_sets().keys()))
def test_device_tree_equals_host_tree(name):
    src, trg, kw = _edge_sets()[name]
    a, b = _plans(src, trg, **kw)
    _same(a, b)


def test_device_tree_at_1m_and_its_setup_time():
    """The headline point set: bit-identical plan, and the tree + binning
    phases on the GPU against the host's."""
    src = W.config2()["src"]
    a, b = _plans(src, pts_max=64)
    _same(a, b)
    ta, tb = a.setup_times(), b.setup_times()
    for _ in range(2):  # again, warm
        a.setup(src)
        b.setup(src)
        ta, tb = a.setup_times(), b.setup_times()
    print("tree+targets device %.1f ms, host %.1f ms; lists device %.1f ms, host %.1f ms; "
          "setup total device %.1f ms, host %.1f ms" % (
              ta["tree"] + ta["targets"], tb["tree"] + tb["targets"], ta["lists"], tb["lists"], ta["total"],
              tb["total"]))
    print("phases device", {k: round(v, 1) for k, v in ta.items() if not k.startswith("ops")})
    print("phases host  ", {k: round(v, 1) for k, v in tb.items() if not k.startswith("ops")})
    # the upload's parts lie inside it (the phase also allocates the handle's I/O buffers)
    assert sum(ta[k] for k in ("upload_geometry", "upload_lists", "upload_operators", "upload_work")) <= ta["upload"] + 1.0


def test_lists_formed_on_first_use():
    """The expanded V lists and the adjoint's inverted lists are formed on
    first use, not by setup: the list-form M2L (FMMG_HADAMARD=list, which
    reads the expanded lists) agrees with the parent-pair form, forward and
    transposed, and the expanded lists read through fmmg_worklist are the same
    whether or not an evaluate formed them first."""
    import os
    import torch
    rng = np.random.default_rng(5)
    src = W.sphere_clusters(120000, rng)
    n = src.shape[0]
    den = torch.from_numpy(rng.normal(size=n)).cuda()
    w = torch.from_numpy(rng.normal(size=n)).cuda()
    a = fmmg.FMM3d(111, np_=6, pts_max=64, device=0)
    a.setup(src)
    old = os.environ.get("FMMG_HADAMARD")
    os.environ["FMMG_HADAMARD"] = "list"
    try:
        b = fmmg.FMM3d(111, np_=6, pts_max=64, device=0)
        b.setup(src)
    finally:
        if old is None:
            del os.environ["FMMG_HADAMARD"]
        else:
            os.environ["FMMG_HADAMARD"] = old
    # the two forms add the same products in different orders: the FP64 gate
    # is the oracle-parity gate
    for prec, tol in ((fmmg.PREC_FP64, 1e-10), (fmmg.PREC_MIXED, 1e-5)):
        va = torch.zeros(n, dtype=torch.float64, device="cuda")
        vb = torch.zeros_like(va)
        a.evaluate_device(den, va, precision=prec)
        b.evaluate_device(den, vb, precision=prec)
        a.sync()
        b.sync()
        rel = float((va - vb).norm() / va.norm())
        assert rel <= tol, (prec, rel)
    ga = torch.zeros(n, dtype=torch.float64, device="cuda")
    gb = torch.zeros_like(ga)
    a.adjoint_device(None, w, ga)
    b.adjoint_device(None, w, gb)
    a.sync()
    b.sync()
    rel = float((ga - gb).norm() / ga.norm())
    assert rel <= 1e-10, rel
    for which in (6, 7):  # a never formed them for an evaluate; b did
        for x, y in zip(a.worklist(which), b.worklist(which)):
            assert (x is None and y is None) or np.array_equal(x, y)


def test_resetup_reuses_device_blocks():
    """A handle set up again keeps its device blocks for the next setup and
    frees the ones nothing reused: growing, shrinking and separate-target
    setups on one handle give what a fresh handle gives, forward, mixed and
    through check() (whose targets are read back from the device)."""
    import torch
    rng = np.random.default_rng(9)
    cases = [(W.uniform(50000, rng), None), (W.sphere_clusters(90000, rng), None),
             (W.uniform(30000, rng), W.uniform(20000, rng)), (W.uniform(50000, rng), None)]
    h = fmmg.FMM3d(111, np_=5, pts_max=48, device=0)
    for src, trg in cases:
        h.setup(src, None, trg)
        g = fmmg.FMM3d(111, np_=5, pts_max=48, device=0)
        g.setup(src, None, trg)
        ns, nt = src.shape[0], (src if trg is None else trg).shape[0]
        den = torch.from_numpy(rng.normal(size=ns)).cuda()
        for prec, tol in ((fmmg.PREC_FP64, 1e-13), (fmmg.PREC_MIXED, 1e-6)):
            vh = torch.zeros(nt, dtype=torch.float64, device="cuda")
            vg = torch.zeros_like(vh)
            h.evaluate_device(den, vh, precision=prec)
            g.evaluate_device(den, vg, precision=prec)
            h.sync()
            g.sync()
            assert float((vh - vg).norm() / vg.norm()) <= tol, prec
        idx = rng.choice(nt, 200, replace=False)
        dh = den.cpu().numpy()
        val = h.evaluate(dh).ravel()
        rh, mh, densh = h.check(dh, val, idx)
        rg, mg, densg = g.check(dh, val, idx)
        # the same targets (a wrong read-back moves them: errors of O(1)); the
        # dense sums add in block order, so they agree to rounding
        assert np.abs(densh - densg).max() <= 1e-12 * np.abs(densg).max()
        assert rh < 1e-4 and abs(rh - rg) <= 1e-9 * max(rg, 1e-12) + 1e-15  # np=5 truncation
