"""CPU checks of the oracle (the FP64 restatement of the reference evaluate()).

The reference holds no golden vectors and cannot be built here, so the oracle
is pinned piece by piece against independent implementations: numpy's FFT for
the FFTW r2c/c2r layout (matmgnt3d_mpi.cpp:302,341,408), numpy's SVD for the
truncated pseudo-inverse (common/vecmatop.cpp:129-164), a numpy restatement of
every kernel formula (kernel3d_mpi.cpp:142-466), structural properties of the
U/V/W/X lists (let3d_mpi.cpp:1637-1768), and end to end the FP64 dense direct
sum used by the reference check() (fmm3d_check_mpi.cpp:122-165).
"""
import numpy as np
import pytest

import oracle as O

KERNELS = (111, 121, 311, 312, 321, 322, 511, 521)


def _unit_normals(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None]


def _numpy_kernel(kt, src, nrm, trg, mu=1.0, ve=0.25):
    """Independent numpy statement of kernel3d_mpi.cpp:152-419, blocks [t][s]."""
    d = trg[:, None, :] - src[None, :, :]
    r2 = (d ** 2).sum(-1)
    r = np.sqrt(r2)
    x, y, z = d[..., 0], d[..., 1], d[..., 2]
    n = nrm[None, :, :]
    rn = (d * n).sum(-1)
    I = np.eye(3)
    with np.errstate(divide="ignore", invalid="ignore"):
        if kt == 111:
            K = (1 / (4 * np.pi) / r)[..., None, None]
        elif kt == 121:
            K = (-1 / (4 * np.pi) / r ** 3 * rn)[..., None, None]
        elif kt in (311, 511, 301):
            if kt == 511:
                G = (3 - 4 * ve) / (16 * np.pi * (1 - ve)) / r / mu
                H = 1 / (16 * np.pi * (1 - ve)) / r ** 3 / mu
            else:
                G = 1 / (8 * np.pi) / r / mu
                H = 1 / (8 * np.pi) / r ** 3 / mu
            K = G[..., None, None] * I + H[..., None, None] * d[..., :, None] * d[..., None, :]
            if kt == 301:
                A = 1 / (4 * np.pi) / r ** 3
                K = np.concatenate([K, (A[..., None] * d)[..., :, None]], axis=-1)
        elif kt == 312:
            K = (1 / (4 * np.pi) / r ** 3)[..., None, None] * d[..., None, :]
        elif kt == 321:
            C = -6 / (8 * np.pi) / r ** 5
            K = (C * rn)[..., None, None] * d[..., :, None] * d[..., None, :]
        elif kt == 322:
            c = mu / (2 * np.pi)
            K = c * (n / r[..., None] ** 3 - 3 * rn[..., None] * d / r[..., None] ** 5)[..., None, :]
        elif kt == 521:
            dc1 = -(1 - 2 * ve) / (8 * np.pi * (1 - ve))
            dc2 = (1 - 2 * ve) / (8 * np.pi * (1 - ve))
            dc3 = -3 / (8 * np.pi * (1 - ve))
            A, B, C = dc1 / r ** 3, dc2 / r ** 3, dc3 / r ** 5
            nn = np.broadcast_to(n, d.shape)
            K = (A[..., None, None] * (rn[..., None, None] * I + nn[..., :, None] * d[..., None, :])
                 + B[..., None, None] * d[..., :, None] * nn[..., None, :]
                 + (C * rn)[..., None, None] * d[..., :, None] * d[..., None, :])
    K = np.where((r < 1e-8)[..., None, None], 0.0, K)
    nt, ns, td, sd = K.shape
    return K.transpose(0, 2, 1, 3).reshape(nt * td, ns * sd)


@pytest.mark.parametrize("kt", KERNELS + (301,))
def test_kernel_matrix_matches_numpy_restatement(kt):
    rng = np.random.default_rng(kt)
    src = rng.random((17, 3))
    trg = rng.random((13, 3))
    trg[0] = src[3]  # coincident pair: the r < 1e-8 block is zero
    nrm = _unit_normals(rng, 17)
    A = O.kernel_matrix(kt, src, nrm, trg, coefs=(1.0, 0.25))
    B = _numpy_kernel(kt, src, nrm, trg, 1.0, 0.25)
    assert A.shape == B.shape
    np.testing.assert_allclose(A, B, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("n,howmany", [(8, 1), (12, 1), (16, 1), (12, 4), (8, 3)])
def test_rfft3_matches_numpy_layout(n, howmany):
    rng = np.random.default_rng(n * 10 + howmany)
    x = rng.normal(size=n ** 3 * howmany)
    X = O.rfft3(x, n, howmany)
    ref = np.fft.rfftn(x.reshape(n, n, n, howmany), axes=(0, 1, 2))  # x axis fastest and halved
    np.testing.assert_allclose(X, ref.ravel(), rtol=1e-12, atol=1e-11)
    back = O.irfft3(X, n, howmany)
    np.testing.assert_allclose(back, x * n ** 3, rtol=1e-12, atol=1e-10)
    ref_back = np.fft.irfftn(ref, s=(n, n, n), axes=(0, 1, 2)) * n ** 3
    np.testing.assert_allclose(back, ref_back.ravel(), rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("np_", [4, 6])
def test_pinv_matches_numpy_svd(np_):
    ue = O.sampos(np_, 1.0)
    uc = O.sampos(np_ + 2, 3.0)
    A = O.kernel_matrix(111, ue, ue, uc)  # the UE -> UC matrix pinv'd by UpwChk2UpwEqu
    eps = 0.1 ** (np_ + 1)
    R = O.pinv(A, eps)
    U, S, Vt = np.linalg.svd(A, full_matrices=False)
    k = int((S >= eps * S[0]).sum())
    Rn = Vt[:k].T @ np.diag(1 / S[:k]) @ U[:, :k].T
    # entries of a pseudo-inverse truncated at eps*s_max agree to about
    # machine eps times the kept condition number (1/eps) between SVD codes
    tol = 1e-16 / eps * 100
    np.testing.assert_allclose(R, Rn, rtol=0, atol=tol * np.abs(Rn).max())
    # Moore-Penrose: A R A = A on the kept subspace
    np.testing.assert_allclose(A @ R @ A, A, rtol=0, atol=1e-12 * np.abs(A).max() / eps)


def test_surfaces_and_grid_sizes():
    # matmgnt3d_mpi.cpp:453,480 and the table of sizes per np
    for np_, ue, uc in ((4, 56, 152), (6, 152, 296), (8, 296, 488)):
        assert O.sampos(np_, 1.0).shape == (ue, 3)
        assert O.sampos(np_ + 2, 3.0).shape == (uc, 3)
        assert O.regpos(np_, 1.0).shape == ((2 * np_) ** 3, 3)
    p = O.sampos(4, 3.0)
    assert np.isclose(np.abs(p).max(), 3.0) and np.isclose(np.abs(p).max(axis=1).min(), 3.0)


def _points(rng, n):
    return rng.random((n, 3))


def test_tree_structure_and_lists():
    rng = np.random.default_rng(7)
    N = 6000
    src = np.concatenate([_points(rng, N // 2), 0.3 + 0.02 * rng.normal(size=(N // 2, 3))])
    src = np.clip(src, 0, 1 - 1e-12)
    o = O.Oracle(111, np_=4, pts_max=40)
    o.setup(src, src, src)
    nd = o.nodes()
    depth, par, chd, src_cnt, trg_cnt = nd[:, 0], nd[:, 4], nd[:, 5], nd[:, 7], nd[:, 8]
    leaf = chd == -1
    assert src_cnt[leaf].sum() == N and trg_cnt[0] == N
    assert (src_cnt[leaf] <= 40).all()
    assert (src_cnt[~leaf][1:] > 40).all()  # non-root interior nodes were split for a reason
    assert not leaf[0]
    for which in range(4):
        ptr, idx = o.lists(which)
        assert (np.diff(ptr) >= 0).all()
    # U and V are symmetric when sources and targets coincide
    for which in (0, 1):
        ptr, idx = o.lists(which)
        pairs = {(a, b) for a in range(len(nd)) for b in idx[ptr[a]:ptr[a + 1]]}
        for a, b in pairs:
            assert (b, a) in pairs
    # V members are same-depth, W deeper, X shallower
    for which, rel in ((1, 0), (2, 1), (3, -1)):
        ptr, idx = o.lists(which)
        for a in range(len(nd)):
            for b in idx[ptr[a]:ptr[a + 1]]:
                assert np.sign(depth[b] - depth[a]) == rel
    # W and X are duals when sources and targets coincide: b in W(a) <=> a in X(b)
    pw, iw = o.lists(2)
    px, ix = o.lists(3)
    W = {(a, int(b)) for a in range(len(nd)) for b in iw[pw[a]:pw[a + 1]]}
    X = {(int(a), b) for b in range(len(nd)) for a in ix[px[b]:px[b + 1]]}
    assert len(W) > 0 and W == X


@pytest.mark.parametrize("kt", KERNELS)
def test_oracle_vs_dense_sum(kt):
    rng = np.random.default_rng(100 + kt)
    N = 3000
    src = _points(rng, N)
    nrm = _unit_normals(rng, N)
    o = O.Oracle(kt, np_=6, pts_max=50, coefs=(1.0, 0.25))
    o.setup(src, nrm, src)
    den = rng.uniform(-1, 1, N * o.sd)
    val = o.evaluate(den)
    ck = rng.choice(N, 150, replace=False)
    ref = O.dense(kt, src, nrm, den, src[ck])
    got = val.reshape(N, o.td)[ck].ravel()
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 5e-5, err


def test_oracle_linear_and_stage_sum():
    rng = np.random.default_rng(3)
    N = 2500
    src = _points(rng, N)
    o = O.Oracle(111, np_=4, pts_max=30)
    o.setup(src, src, src)
    a, b = rng.normal(size=N), rng.normal(size=N)
    va, vb, vab = o.evaluate(a), o.evaluate(b), o.evaluate(2 * a - 3 * b)
    np.testing.assert_allclose(vab, 2 * va - 3 * vb, rtol=0, atol=1e-12 * np.abs(vab).max())
    # near-field stages are additive on their own
    s = sum(o.evaluate(a, stages=m) for m in (O.STAGE_U, O.STAGE_W | O.STAGE_UP))
    both = o.evaluate(a, stages=O.STAGE_U | O.STAGE_W | O.STAGE_UP)
    np.testing.assert_allclose(s, both, rtol=0, atol=1e-12 * np.abs(both).max())


def test_separate_targets_binned_into_source_tree():
    rng = np.random.default_rng(11)
    src = _points(rng, 2000)
    trg = _points(rng, 700)
    o = O.Oracle(111, np_=4, pts_max=30)
    o.setup(src, src, trg)
    den = rng.normal(size=2000)
    val = o.evaluate(den)
    ref = O.dense(111, src, src, den, trg)
    assert np.linalg.norm(val - ref) / np.linalg.norm(ref) < 1e-3


@pytest.mark.parametrize("np_", [6, 8])
def test_reordering_floor_of_the_reference_arithmetic(np_):
    """The FP64 evaluate() of the reference sums every operator GEMV in BLAS
    column order.  Summing the columns of any one operator class in reverse
    (an equally valid order) moves the result by the reordering floor that the
    GPU/oracle parity gate allows for: rounding upstream of a C2E
    pseudo-inverse (cutoff 0.1^(np+1), matmgnt3d_mpi.cpp:37-40) is amplified,
    ~1e-11 at np=6 and ~1e-9 at np=8, from M2M and L2L as much as from the
    pseudo-inverses themselves."""
    rng = np.random.default_rng(20261203 + np_)
    n = 5000
    src = rng.random((n, 3))
    den = rng.uniform(-1, 1, n)
    o = O.Oracle(111, np_=np_, pts_max=40, nthreads=8)
    o.setup(src, src, src)
    a = o.evaluate(den)
    floors = {}
    for mask in (O.Oracle.GEMV_UP_C2E, O.Oracle.GEMV_M2M, O.Oracle.GEMV_DN_C2E, O.Oracle.GEMV_L2L, True):
        o.set_gemv_order(mask)
        floors[mask] = np.linalg.norm(o.evaluate(den) - a) / np.linalg.norm(a)
    o.set_gemv_order(False)
    assert np.array_equal(o.evaluate(den), a)  # the reference order again, bit for bit
    if np_ <= 6:
        assert max(floors.values()) < 1e-10
    else:
        assert min(floors.values()) > 1e-10  # every class alone reaches it
        assert max(floors.values()) < 1e-8
