"""GPU parity: the plain FP64 CUDA evaluate vs the CPU oracle, through the C ABI.

Gate (north star): relative L2 <= 1e-10 on the same tree, operators and inputs.
The oracle is handed the library's operator tables for that gate; with each
side's own tables the two pseudo-inverses come from different SVD codes and the
bound is looser (tested separately).  Accuracy against the FP64 dense sum (the
reference check(), fmm3d_mpi/fmm3d_check_mpi.cpp:122-165) is stated per case.
"""
import numpy as np
import pytest

import fmmg
import oracle as O
from gpu_common import SEED, gpu_eval, points, rel_l2, share_operators, unit_normals

pytestmark = pytest.mark.gpu

PARITY = 1e-10
KERNELS = (111, 121, 311, 312, 321, 322, 511, 521)


def _case(kt, np_, n, kind="uniform", pts=40, seed=0, sep_targets=0):
    rng = np.random.default_rng(SEED + seed)
    src = points(kind, n, rng)
    nrm = unit_normals(rng, n)
    trg = rng.random((sep_targets, 3)) if sep_targets else src
    lib = fmmg.FMM3d(kt, np_=np_, pts_max=pts)
    lib.setup(src, nrm, trg)
    orc = O.Oracle(kt, np_=np_, pts_max=pts)
    orc.setup(src, nrm, trg)
    share_operators(lib, orc)
    den = rng.uniform(-1, 1, n * lib.sd)
    return lib, orc, src, nrm, trg, den


@pytest.mark.parametrize("kt", KERNELS)
def test_fp64_parity_all_kernels_np4(kt):
    lib, orc, *_, den = _case(kt, 4, 6000, "sphere_clusters", pts=30, seed=kt)
    g = gpu_eval(lib, den)
    c = orc.evaluate(den)
    assert rel_l2(g, c) <= PARITY


def parity_tol(np_):
    # The C2E pseudo-inverse keeps singular values down to 0.1^(np+1) of the
    # largest (matmgnt3d_mpi.cpp:37-40), so two FP64 codes that sum in a
    # different order agree to about eps_mach * 10^(np+1) at worst: within
    # 1e-10 up to np = 7; at np = 8 (cutoff 1e-9) the bound is 1e-8.
    return PARITY if np_ <= 7 else 1e-8


@pytest.mark.parametrize("kt,np_", [(111, 6), (111, 8), (121, 6), (321, 6), (511, 6), (312, 5), (111, 3), (111, 7)])
def test_fp64_parity_np(kt, np_):
    lib, orc, *_, den = _case(kt, np_, 5000, "uniform", pts=40, seed=np_)
    g = gpu_eval(lib, den)
    c = orc.evaluate(den)
    assert rel_l2(g, c) <= parity_tol(np_)


@pytest.mark.parametrize("stages", [O.STAGE_U, O.STAGE_W | O.STAGE_UP, O.STAGE_X, O.STAGE_X | O.STAGE_DOWN,
                                    O.STAGE_UP | O.STAGE_V | O.STAGE_DOWN, O.STAGE_UP | O.STAGE_DOWN])
def test_stage_parity(stages):
    lib, orc, *_, den = _case(111, 4, 8000, "sphere_clusters", pts=20, seed=3)
    g = gpu_eval(lib, den, stages)
    c = orc.evaluate(den, stages=stages)
    if np.linalg.norm(c) == 0:
        assert np.linalg.norm(g) == 0
    else:
        assert rel_l2(g, c) <= PARITY


def test_config1_laplace_65536_np4():
    """Config 1: 65,536 uniform points, Laplace S, np=4, ptsMax=150, check at 1,000 targets."""
    rng = np.random.default_rng(SEED + 1)
    n = 65536
    src = rng.random((n, 3))
    den = rng.uniform(-1, 1, n)
    lib = fmmg.FMM3d(111, np_=4, pts_max=150, max_level=30)
    lib.setup(src)
    orc = O.Oracle(111, np_=4, pts_max=150, max_level=30, nthreads=8)
    orc.setup(src, src, src)
    share_operators(lib, orc)
    g = lib.evaluate(den).ravel()  # host-buffer path through the C ABI
    c = orc.evaluate(den)
    assert rel_l2(g, c) <= PARITY
    idx = rng.choice(n, 1000, replace=False)
    err, mx, dense = lib.check(den, g, idx)
    ref = O.dense(111, src, src, den, src[idx], nthreads=8)
    np.testing.assert_allclose(dense.ravel(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    assert err < 1e-3  # np=4 is the reference's "low accuracy" setting


def test_own_operators_close_to_oracle_own_operators():
    rng = np.random.default_rng(SEED + 7)
    n = 6000
    src = points("uniform", n, rng)
    lib = fmmg.FMM3d(111, np_=6, pts_max=40)
    lib.setup(src)
    orc = O.Oracle(111, np_=6, pts_max=40)
    orc.setup(src, src, src)
    den = rng.normal(size=n)
    # two SVD codes: pinv entries differ at eps_mach / cutoff, far less after the far-field sum
    assert rel_l2(gpu_eval(lib, den), orc.evaluate(den)) <= 1e-8


def test_separate_targets_and_dense_error():
    lib, orc, src, nrm, trg, den = _case(111, 6, 7000, "uniform", pts=50, seed=11, sep_targets=3000)
    g = gpu_eval(lib, den)
    assert rel_l2(g, orc.evaluate(den)) <= PARITY
    idx = np.arange(0, 3000, 7)
    err, _, _ = lib.check(den, g, idx)
    assert err < 1e-5


def test_multiple_rhs_and_linearity():
    import torch
    lib, orc, *_, den = _case(111, 4, 5000, "uniform", pts=40, seed=13)
    rng = np.random.default_rng(5)
    k = 3
    D = rng.normal(size=(k, lib.ns))
    d = torch.from_numpy(D).cuda()
    out = torch.zeros(k, lib.nt, dtype=torch.float64, device="cuda")
    lib.evaluate_device(d, out, k=k)
    torch.cuda.synchronize()
    V = out.cpu().numpy()
    for r in range(k):
        assert rel_l2(V[r], gpu_eval(lib, D[r])) <= 1e-14
    comb = gpu_eval(lib, 2 * D[0] - 0.5 * D[1])
    assert rel_l2(comb, 2 * V[0] - 0.5 * V[1]) <= 1e-12


def test_edge_cases():
    # a single source: the root is split into 8 leaves, only the U-list acts
    lib = fmmg.FMM3d(111, np_=4, pts_max=10)
    lib.setup(np.array([[0.2, 0.3, 0.4]]), trg=np.array([[0.2, 0.3, 0.4], [0.9, 0.9, 0.9]]))
    v = lib.evaluate(np.array([2.0])).ravel()
    assert v[0] == 0.0  # coincident pair is zero (kernel3d_mpi.cpp:160)
    assert abs(v[1] - 2.0 / (4 * np.pi * np.linalg.norm([0.7, 0.6, 0.5]))) < 1e-14
    # duplicate points down to max_level and points on the box faces
    rng = np.random.default_rng(2)
    src = np.concatenate([np.full((60, 3), 0.25), rng.random((500, 3)), [[0, 0, 0], [1, 1, 1], [1, 0, 0.5]]])
    lib = fmmg.FMM3d(111, np_=4, pts_max=20, max_level=6)
    lib.setup(src)
    orc = O.Oracle(111, np_=4, pts_max=20, max_level=6)
    orc.setup(src, src, src)
    share_operators(lib, orc)
    den = rng.normal(size=len(src))
    assert rel_l2(gpu_eval(lib, den), orc.evaluate(den)) <= PARITY
    # no targets
    lib = fmmg.FMM3d(111, np_=4, pts_max=20)
    lib.setup(rng.random((100, 3)), trg=np.zeros((0, 3)))
    assert lib.evaluate(rng.normal(size=100)).size == 0
